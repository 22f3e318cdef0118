"""CPU oracle for the shell spectra of HIT snapshots (NumPy, FP64).

TEST INFRASTRUCTURE ONLY.  Nothing under ``hit_solver_b200/`` imports this
module.  Only ``tests/`` and the CPU legs of ``bench.py`` may call it, and
there only as the checker (or as the timed CPU baseline).

A restatement, in my own code, of the arithmetic of
``HIT2DSpectra.compute`` in the reference's ``OOP/postprocess/spectra.py``
(lines 48-149, with ``_fluctuations`` at 199-210 and
``_cutoff_pileup_ratio`` at 212-222).  It works on arrays, not on snapshot
files: the file selection (time window, stride) is plain host logic of the
package mirror.  Pinned against the reference's own output on snapshots that
the reference's ``run_simulation`` wrote (``tests/golden/spectra_*.npz``,
made by ``tests/golden/make_golden.py``; checked in
``tests/test_oracle_golden.py``).
"""

from __future__ import annotations

import numpy as np


def fluctuations(rho, u, v, kind: str):
    """Velocity fluctuations about the Reynolds (plain) or Favre
    (density-weighted) mean, spectra.py:199-210."""
    if kind == "favre":
        mass = float(np.mean(rho))
        um = float(np.mean(rho * u) / mass)
        vm = float(np.mean(rho * v) / mass)
    elif kind == "reynolds":
        um, vm = float(np.mean(u)), float(np.mean(v))
    else:
        raise ValueError(kind)
    return u - um, v - vm


def shell_geometry(nx: int, ny: int, dx: float, dy: float):
    """(kx grid, ky grid, shell index of every mode, dk, last shell),
    spectra.py:90-99: wavenumbers 2 pi fftfreq, dk the smaller fundamental,
    shells rint(|k| / dk)."""
    kx = 2.0 * np.pi * np.fft.fftfreq(nx, d=dx)
    ky = 2.0 * np.pi * np.fft.fftfreq(ny, d=dy)
    KX = np.broadcast_to(kx[None, :], (ny, nx))
    KY = np.broadcast_to(ky[:, None], (ny, nx))
    dk = min(2.0 * np.pi / (nx * dx), 2.0 * np.pi / (ny * dy))
    shell = np.rint(np.sqrt(KX ** 2 + KY ** 2) / dk).astype(np.int64)
    return KX, KY, shell, dk, min(nx, ny) // 2


def snapshot_shells(x, y, rho, u, v, kind: str = "reynolds"):
    """Shell sums of one snapshot, spectra.py:84-121: the energy of the
    sqrt(rho)-weighted fluctuations and the enstrophy of the spectral
    vorticity of the plain fluctuations, each 1/2 |.|^2 / (nx ny)^2 per mode.
    Returns (k, energy[last + 1], enstrophy[last + 1])."""
    up, vp = fluctuations(rho, u, v, kind)
    ny, nx = rho.shape
    KX, KY, shell, dk, last = shell_geometry(nx, ny, float(x[1] - x[0]), float(y[1] - y[0]))
    scale = float(nx * ny) ** 2
    root = np.sqrt(rho)
    a, b = np.fft.fft2(root * up), np.fft.fft2(root * vp)
    e_mode = 0.5 * (np.abs(a) ** 2 + np.abs(b) ** 2) / scale
    uh, vh = np.fft.fft2(up), np.fft.fft2(vp)
    z_mode = 0.5 * np.abs(1j * (KX * vh - KY * uh)) ** 2 / scale
    idx = shell.ravel()
    keep = idx <= last
    energy = np.zeros(last + 1)
    enstrophy = np.zeros(last + 1)
    np.add.at(energy, idx[keep], e_mode.ravel()[keep])
    np.add.at(enstrophy, idx[keep], z_mode.ravel()[keep])
    return dk * np.arange(last + 1), energy, enstrophy


def pileup_ratio(values) -> float:
    """Mean of the last tenth (at least 3) of the nonzero shells over the mean
    of the tenth before it; 0 when too few shells or a negligible tail,
    spectra.py:212-222."""
    tail = np.asarray(values)[1:]
    w = max(3, tail.size // 10)
    if tail.size < 2 * w:
        return 0.0
    before = float(np.mean(tail[-2 * w:-w]))
    last = float(np.mean(tail[-w:]))
    if float(np.sum(tail[-w:])) < 1.0e-8 * float(np.sum(tail)):
        return 0.0
    return last / max(before, np.finfo(float).tiny)


def spectra_summary(snapshots, kind: str = "reynolds") -> dict:
    """Statistics over the selected snapshots, spectra.py:123-149.
    ``snapshots``: iterable of (time, x, y, rho, u, v)."""
    es, zs, times, k = [], [], [], None
    for t, x, y, rho, u, v in snapshots:
        k, e, z = snapshot_shells(x, y, rho, u, v, kind)
        es.append(e)
        zs.append(z)
        times.append(float(t))
    E, Z = np.stack(es), np.stack(zs)
    em, zm = E.mean(axis=0), Z.mean(axis=0)
    return {"k": k, "energy_mean": em, "energy_std": E.std(axis=0), "enstrophy_mean": zm,
            "enstrophy_std": Z.std(axis=0), "number_of_snapshots": len(es),
            "selected_time_interval": (times[0], times[-1]),
            "high_k_energy_ratio": pileup_ratio(em), "high_k_enstrophy_ratio": pileup_ratio(zm)}
