"""Shell-averaged kinetic-energy and enstrophy spectra on the device.

Mirrors ``HIT2DSpectra`` of the reference (``OOP/postprocess/spectra.py``):
same constructor, ``compute()`` result, ``save()`` keys, exceptions and
warnings.  The per-snapshot work (fluctuations, four 2-D transforms, shell
binning of the mode energies and enstrophies) runs for all selected
snapshots at once on the GPU:

* ``hitb200_spectra_fields`` / ``hitb200_spectra_state_fields`` (CUDA) form
  sqrt(rho) u', sqrt(rho) v', u', v' of every snapshot;
* ``hitb200_rfft2`` (the library's mixed-radix line transforms) gives their
  half spectra, enough for real fields;
* ``hitb200_spectra_shells`` (CUDA) bins the modes into shells in a fixed
  order.

The statistics over snapshots (mean, standard deviation, pile-up ratios) are
a few hundred numbers and stay on the host, in NumPy, as in the reference.
:func:`shell_spectra` and :func:`state_shell_spectra` expose the batched
device reduction for device-resident fields or states (ensemble statistics of
running solves without writing snapshots).
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from .. import _lib, core


@dataclass
class SpectrumResults2D:
    """Result of :meth:`HIT2DSpectra.compute` (spectra.py:11-21)."""

    k: np.ndarray
    energy_mean: np.ndarray
    energy_std: np.ndarray
    enstrophy_mean: np.ndarray
    enstrophy_std: np.ndarray
    number_of_snapshots: int
    selected_time_interval: tuple[float, float]
    high_k_energy_ratio: float
    high_k_enstrophy_ratio: float


def _fields3(t: torch.Tensor, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise TypeError(f"{name} must be a torch CUDA tensor")
    if t.dim() == 2:
        t = t.unsqueeze(0)
    if t.dim() != 3:
        raise ValueError(f"{name} must have shape [n_snap, ny, nx] or [ny, nx]")
    return t.to(torch.float64).contiguous()


def _shells(fields: torch.Tensor, nx: int, ny: int, dx: float, dy: float, ws: torch.Tensor):
    lib = _lib.load()
    n = fields.shape[0]
    # [n, 4, ny, nx // 2 + 1] complex128: the library's line transforms
    spec = torch.empty((n, 4, ny, nx // 2 + 1), dtype=torch.complex128, device=fields.device)
    fws = torch.empty(int(lib.hitb200_rfft2_workspace_bytes(nx, ny)), dtype=torch.uint8,
                      device=fields.device)
    _lib.check(lib.hitb200_rfft2(fields.data_ptr(), 4 * n, nx, ny, spec.data_ptr(), fws.data_ptr(),
                                 fws.numel(), core.stream_handle()))
    ns = min(nx, ny) // 2 + 1
    energy = torch.empty((n, ns), dtype=torch.float64, device=fields.device)
    enstrophy = torch.empty_like(energy)
    _lib.check(lib.hitb200_spectra_shells(spec.data_ptr(), n, nx, ny, float(dx), float(dy),
                                          energy.data_ptr(), enstrophy.data_ptr(), ws.data_ptr(),
                                          ws.numel(), core.stream_handle()))
    dk = min(2.0 * np.pi / (nx * dx), 2.0 * np.pi / (ny * dy))
    return dk * np.arange(ns), energy, enstrophy


def _workspace(n: int, nx: int, ny: int, device) -> torch.Tensor:
    size = int(_lib.load().hitb200_spectra_workspace_bytes(n, nx, ny))
    if size == 0:
        raise ValueError("spectra: need at least one snapshot of at least 2 x 2 cells")
    return torch.empty(size, dtype=torch.uint8, device=device)


def _kind(fluctuation_type: str) -> int:
    kind = fluctuation_type.lower()
    if kind not in {"reynolds", "favre"}:
        raise ValueError("fluctuation_type must be 'reynolds' or 'favre'")
    return 1 if kind == "favre" else 0


def shell_spectra(rho, u, v, dx: float, dy: float, fluctuation_type: str = "reynolds"):
    """Shell spectra of snapshots given as primitive fields.

    rho, u, v: CUDA tensors [n_snap, ny, nx] (or one [ny, nx] snapshot), one
    grid with spacings dx, dy.  Returns (k, energy, enstrophy): the shell
    wavenumbers dk * arange(ns) (NumPy) and the per-snapshot shell sums,
    CUDA float64 [n_snap, ns], ns = min(nx, ny) // 2 + 1 (spectra.py:84-121).
    """
    core.require_cuda()
    favre = _kind(fluctuation_type)
    rho, u, v = _fields3(rho, "rho"), _fields3(u, "u"), _fields3(v, "v")
    if u.shape != rho.shape or v.shape != rho.shape:
        raise ValueError("rho, u and v must have the same shape")
    n, ny, nx = rho.shape
    ws = _workspace(n, nx, ny, rho.device)
    fields = torch.empty((n, 4, ny, nx), dtype=torch.float64, device=rho.device)
    _lib.check(_lib.load().hitb200_spectra_fields(rho.data_ptr(), u.data_ptr(), v.data_ptr(), n, nx,
                                                  ny, favre, fields.data_ptr(), ws.data_ptr(),
                                                  ws.numel(), core.stream_handle()))
    return _shells(fields, nx, ny, dx, dy, ws)


def state_shell_spectra(q, dx: float, dy: float, fluctuation_type: str = "reynolds"):
    """Shell spectra of conservative states [n_snap, 4, ny, nx] (or one
    [4, ny, nx]) with the primitives of ``primitive_from_conservative``
    (density floor 1e-10), as the reference's snapshots store them."""
    core.require_cuda()
    favre = _kind(fluctuation_type)
    if not isinstance(q, torch.Tensor) or q.device.type != "cuda":
        raise TypeError("q must be a torch CUDA tensor")
    if q.dim() == 3:
        q = q.unsqueeze(0)
    if q.dim() != 4 or q.shape[1] != 4:
        raise ValueError("q must have shape [n_snap, 4, ny, nx] or [4, ny, nx]")
    q = q.to(torch.float64).contiguous()
    n, _, ny, nx = q.shape
    ws = _workspace(n, nx, ny, q.device)
    fields = torch.empty((n, 4, ny, nx), dtype=torch.float64, device=q.device)
    _lib.check(_lib.load().hitb200_spectra_state_fields(q.data_ptr(), n, nx, ny, favre,
                                                        fields.data_ptr(), ws.data_ptr(),
                                                        ws.numel(), core.stream_handle()))
    return _shells(fields, nx, ny, dx, dy, ws)


def _cutoff_pileup_ratio(values: np.ndarray) -> float:
    """Tail mean over the mean of the band before it (spectra.py:212-222)."""
    nonzero = values[1:]
    width = max(3, nonzero.size // 10)
    if nonzero.size < 2 * width:
        return 0.0
    band = float(np.mean(nonzero[-2 * width:-width]))
    tail = float(np.mean(nonzero[-width:]))
    if float(np.sum(nonzero[-width:])) < 1.0e-8 * float(np.sum(nonzero)):
        return 0.0
    return tail / max(band, np.finfo(float).tiny)


class HIT2DSpectra:
    """Shell-averaged kinetic-energy and enstrophy spectra from HIT2D
    snapshots (``hit2d_step*.npz`` of a run directory), spectra.py:24-46."""

    def __init__(self, run_dir, fluctuation_type: str = "reynolds", start_time=None,
                 end_time=None, stride: int = 1, output_dir=None) -> None:
        self.run_dir = Path(run_dir)
        self.fluctuation_type = fluctuation_type.lower()
        if self.fluctuation_type not in {"reynolds", "favre"}:
            raise ValueError("fluctuation_type must be 'reynolds' or 'favre'")
        if stride <= 0:
            raise ValueError("stride must be positive")
        self.start_time = start_time
        self.end_time = end_time
        self.stride = stride
        self.output_dir = Path(output_dir) if output_dir is not None else self.run_dir / "postprocess"
        self.results: SpectrumResults2D | None = None

    def _select(self):
        """(time, path) of the snapshots in the window, every stride-th one
        (spectra.py:48-76)."""
        paths = sorted(self.run_dir.glob("hit2d_step*.npz"))
        if not paths:
            raise FileNotFoundError(f"No HIT2D snapshots found in {self.run_dir}")
        chosen = []
        for path in paths:
            with np.load(path) as data:
                t = float(data["time"])
            if self.start_time is not None and t < self.start_time:
                continue
            if self.end_time is not None and t > self.end_time:
                continue
            chosen.append((t, path))
        chosen = chosen[:: self.stride]
        if not chosen:
            raise ValueError("No snapshots are available in the selected spectral interval")
        if len(chosen) < 5:
            warnings.warn("Few snapshots selected for spectral averaging", RuntimeWarning)
        return chosen

    def compute(self) -> SpectrumResults2D:
        chosen = self._select()
        core.require_cuda()
        # snapshots grouped by grid; one batched device pass per group
        groups: dict = {}
        for pos, (_t, path) in enumerate(chosen):
            with np.load(path) as data:
                x = np.asarray(data["x"], dtype=float)
                y = np.asarray(data["y"], dtype=float)
                fields = [np.asarray(data[k], dtype=float) for k in ("rho", "u", "v")]
            key = (x.size, y.size, float(x[1] - x[0]), float(y[1] - y[0]))
            groups.setdefault(key, []).append((pos, fields))
        energy = [None] * len(chosen)
        enstrophy = [None] * len(chosen)
        k_shell = None  # the last snapshot's shells, as in the reference
        for key, members in groups.items():
            nx, ny, dx, dy = key
            host = [torch.from_numpy(np.stack([m[1][c] for m in members])).pin_memory()
                    for c in range(3)]
            dev = [h.to("cuda", non_blocking=True) for h in host]
            k, e, z = shell_spectra(dev[0], dev[1], dev[2], dx, dy, self.fluctuation_type)
            e, z = e.cpu().numpy(), z.cpu().numpy()
            for row, (pos, _f) in enumerate(members):
                energy[pos], enstrophy[pos] = e[row], z[row]
            if members[-1][0] == len(chosen) - 1:
                k_shell = k
        energy_stack = np.stack(energy)
        enstrophy_stack = np.stack(enstrophy)
        energy_mean = np.mean(energy_stack, axis=0)
        enstrophy_mean = np.mean(enstrophy_stack, axis=0)
        hk_e = _cutoff_pileup_ratio(energy_mean)
        hk_z = _cutoff_pileup_ratio(enstrophy_mean)
        if hk_e > 2.0:
            warnings.warn("Kinetic-energy spectrum may be piling up near k_max", RuntimeWarning)
        if hk_z > 2.0:
            warnings.warn("Enstrophy spectrum may be piling up near k_max", RuntimeWarning)
        times = [t for t, _p in chosen]
        self.results = SpectrumResults2D(
            k=k_shell, energy_mean=energy_mean, energy_std=np.std(energy_stack, axis=0),
            enstrophy_mean=enstrophy_mean, enstrophy_std=np.std(enstrophy_stack, axis=0),
            number_of_snapshots=len(chosen),
            selected_time_interval=(float(times[0]), float(times[-1])),
            high_k_energy_ratio=hk_e, high_k_enstrophy_ratio=hk_z)
        return self.results

    def save(self, output_path=None) -> Path:
        """The reference's ``spectra_diagnostics.npz`` keys (spectra.py:151-168)."""
        r = self._require_results()
        path = Path(output_path) if output_path is not None else self.run_dir / "spectra_diagnostics.npz"
        path.parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(
            path, k=r.k, energy_mean=r.energy_mean, energy_std=r.energy_std,
            enstrophy_mean=r.enstrophy_mean, enstrophy_std=r.enstrophy_std,
            number_of_snapshots=np.asarray(r.number_of_snapshots),
            selected_time_interval=np.asarray(r.selected_time_interval),
            high_k_energy_ratio=np.asarray(r.high_k_energy_ratio),
            high_k_enstrophy_ratio=np.asarray(r.high_k_enstrophy_ratio),
            fluctuation_type=np.asarray(self.fluctuation_type))
        return path

    def plot(self, output_path=None):
        """Plotting is not part of this backend: the result is the reference's
        SpectrumResults2D, so the reference's own ``HIT2DSpectra.plot`` draws
        it (assign it to that object's ``results``)."""
        raise NotImplementedError("plotting stays with the reference's HIT2DSpectra.plot")

    def _require_results(self) -> SpectrumResults2D:
        if self.results is None:
            raise RuntimeError("Call compute() before save() or plot()")
        return self.results


__all__ = ["HIT2DSpectra", "SpectrumResults2D", "shell_spectra", "state_shell_spectra"]
