"""Shell spectra (HIT2DSpectra, OOP/postprocess/spectra.py:48-149) on the device.

GPU tests: the package mirror over snapshot files against the reference's own
results (tests/golden/spectra_*.npz), the batched device reduction against
the oracle on non-square, odd and 512^2 grids, the conservative-state entry
point, determinism, and Parseval's identity on a 64-snapshot 512^2 batch.
CPU tests: argument checks of the C ABI and of the mirror's constructor.
"""

import ctypes
import math
import warnings
from pathlib import Path

import numpy as np
import pytest
import torch

from hit_solver_b200 import _lib
from oracle import spectra_oracle as SO

G = Path(__file__).resolve().parent / "golden"
SETTINGS = (("reynolds", "reynolds", None, None, 1), ("favre", "favre", None, None, 1),
            ("window", "reynolds", 0.02, 0.07, 2))
# FP64 sums in another order than NumPy's: 1e-12 of the largest shell
ATOL_REL = 1e-12


def _close(got, want, name):
    want = np.asarray(want)
    tol = ATOL_REL * max(float(np.max(np.abs(want))), 1e-300)
    err = float(np.max(np.abs(np.asarray(got) - want)))
    assert err <= tol, (name, err, tol)


def _write_snapshots(d, out: Path):
    for i in range(d["time"].size):
        np.savez_compressed(out / f"hit2d_step{int(d['step'][i]):07d}.npz", step=int(d["step"][i]),
                            time=float(d["time"][i]), x=d["x"], y=d["y"], rho=d["rho"][i],
                            u=d["u"][i], v=d["v"][i])


def _random_fields(n_snap, nx, ny, seed, kmax=None):
    """Random primitive fields (density 0.6..1.4; velocity: a few random
    modes plus white noise) on a 2 pi x 2 pi grid."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) * 2 * np.pi / nx
    y = (np.arange(ny) + 0.5) * 2 * np.pi / ny
    X, Y = np.meshgrid(x, y)
    out = []
    for _ in range(n_snap):
        f = []
        for c in range(3):
            acc = np.zeros((ny, nx))
            for _m in range(12):
                kx, ky = rng.integers(-(kmax or nx // 2), (kmax or nx // 2) + 1, size=2)
                acc += rng.normal() * np.cos(kx * X + ky * Y + rng.uniform(0, 2 * np.pi))
            f.append(acc)
        rho = 1.0 + 0.4 * np.tanh(f[0] / 4)
        # white noise: every mode, the Nyquist row and column included
        out.append((rho, 0.3 + 0.2 * f[1] + 0.05 * rng.normal(size=(ny, nx)),
                    -0.1 + 0.2 * f[2] + 0.05 * rng.normal(size=(ny, nx))))
    rho, u, v = (np.stack([o[c] for o in out]) for c in range(3))
    return x, y, rho, u, v


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["32x24", "25x20"])
def test_mirror_matches_reference_results(tag, tmp_path):
    from hit_solver_b200.postprocess import HIT2DSpectra

    d = np.load(G / f"spectra_{tag}.npz")
    _write_snapshots(d, tmp_path)
    for name, kind, t0, t1, stride in SETTINGS:
        with warnings.catch_warnings(record=True) as caught:
            warnings.simplefilter("always")
            r = HIT2DSpectra(tmp_path, fluctuation_type=kind, start_time=t0, end_time=t1,
                             stride=stride).compute()
        got_w = [str(w.message) for w in caught] or [""]
        assert got_w == list(d[f"{name}_warnings"]), (name, got_w)
        assert r.number_of_snapshots == int(d[f"{name}_n"])
        np.testing.assert_array_equal(np.asarray(r.selected_time_interval), d[f"{name}_interval"])
        np.testing.assert_allclose(r.k, d[f"{name}_k"], rtol=1e-15)
        for key in ("energy_mean", "energy_std", "enstrophy_mean", "enstrophy_std"):
            _close(getattr(r, key), d[f"{name}_{key}"], f"{name} {key}")
        for key, gk in (("high_k_energy_ratio", "hk_energy"), ("high_k_enstrophy_ratio", "hk_enstrophy")):
            assert getattr(r, key) == pytest.approx(float(d[f"{name}_{gk}"]), rel=1e-9)


@pytest.mark.gpu
def test_mirror_save_keys(tmp_path):
    from hit_solver_b200.postprocess import HIT2DSpectra

    d = np.load(G / "spectra_32x24.npz")
    _write_snapshots(d, tmp_path)
    s = HIT2DSpectra(tmp_path, fluctuation_type="favre")
    s.compute()
    with np.load(s.save()) as f:
        assert sorted(f.files) == sorted([
            "k", "energy_mean", "energy_std", "enstrophy_mean", "enstrophy_std",
            "number_of_snapshots", "selected_time_interval", "high_k_energy_ratio",
            "high_k_enstrophy_ratio", "fluctuation_type"])
        assert str(f["fluctuation_type"]) == "favre"


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,kind", [(96, 80, "reynolds"), (63, 50, "favre"),
                                        (128, 128, "favre"), (512, 512, "reynolds")])
def test_batched_shells_match_oracle(nx, ny, kind):
    from hit_solver_b200.postprocess import shell_spectra

    n = 2 if nx == 512 else 5
    x, y, rho, u, v = _random_fields(n, nx, ny, seed=nx + ny)
    t = [torch.from_numpy(a).cuda() for a in (rho, u, v)]
    k, e, z = shell_spectra(*t, float(x[1] - x[0]), float(y[1] - y[0]), kind)
    e, z = e.cpu().numpy(), z.cpu().numpy()
    for s in range(n):
        kw, ew, zw = SO.snapshot_shells(x, y, rho[s], u[s], v[s], kind)
        np.testing.assert_allclose(k, kw, rtol=1e-15)
        _close(e[s], ew, f"energy {s}")
        _close(z[s], zw, f"enstrophy {s}")


@pytest.mark.gpu
def test_state_entry_point_and_determinism():
    from hit_solver_b200.postprocess import shell_spectra, state_shell_spectra

    x, y, rho, u, v = _random_fields(3, 64, 48, seed=3)
    rho[0, 0, 0] = -1.0  # below the density floor: primitive_from_conservative floors it
    q = np.stack([rho, rho * u, rho * v, 2.5 + 0.5 * rho * (u * u + v * v)], axis=1)
    dx, dy = float(x[1] - x[0]), float(y[1] - y[0])
    qd = torch.from_numpy(q).cuda()
    k, e1, z1 = state_shell_spectra(qd, dx, dy, "favre")
    _, e2, z2 = state_shell_spectra(qd, dx, dy, "favre")
    assert torch.equal(e1, e2) and torch.equal(z1, z2)  # fixed-order sums
    r = np.maximum(q[:, 0], 1e-10)
    _, ew, zw = shell_spectra(torch.from_numpy(r).cuda(), torch.from_numpy(q[:, 1] / r).cuda(),
                              torch.from_numpy(q[:, 2] / r).cuda(), dx, dy, "favre")
    _close(e1.cpu().numpy(), ew.cpu().numpy(), "energy")
    _close(z1.cpu().numpy(), zw.cpu().numpy(), "enstrophy")


@pytest.mark.gpu
def test_parseval_on_64_snapshots_512():
    """Band-limited fields (|k| <= 40, every mode inside the last shell): the
    shells of each snapshot sum to 1/2 mean(rho (u'^2 + v'^2)) (Parseval)."""
    from hit_solver_b200.postprocess import shell_spectra

    n, N = 64, 512
    gen = torch.Generator(device="cuda").manual_seed(11)
    xs = torch.arange(N, device="cuda", dtype=torch.float64) * (2 * math.pi / N)
    X, Y = xs[None, :], xs[:, None]

    def field(amp):
        acc = torch.zeros((n, N, N), device="cuda", dtype=torch.float64)
        for _ in range(6):
            kx = torch.randint(-28, 29, (n, 1, 1), generator=gen, device="cuda").double()
            ky = torch.randint(-28, 29, (n, 1, 1), generator=gen, device="cuda").double()
            ph = 2 * math.pi * torch.rand((n, 1, 1), generator=gen, device="cuda", dtype=torch.float64)
            acc += torch.cos(kx * X + ky * Y + ph)
        return amp * acc

    rho = 1.0 + 0.0 * field(1.0)
    u, v = field(0.1), field(0.1)
    k, e, z = shell_spectra(rho, u, v, 2 * math.pi / N, 2 * math.pi / N, "reynolds")
    up = u - u.mean(dim=(1, 2), keepdim=True)
    vp = v - v.mean(dim=(1, 2), keepdim=True)
    want = 0.5 * (rho * (up * up + vp * vp)).mean(dim=(1, 2))
    got = e.sum(dim=1)
    assert torch.allclose(got, want, rtol=1e-12, atol=0.0)
    assert e.shape == (n, N // 2 + 1) and bool((e >= 0).all()) and bool((z >= 0).all())


# ---------------------------------------------------------------- CPU ----------
def test_spectra_abi_rejects_bad_arguments():
    lib = _lib.load()
    buf = ctypes.create_string_buffer(64)
    p = ctypes.addressof(buf)
    assert lib.hitb200_spectra_workspace_bytes(0, 8, 8) == 0
    assert lib.hitb200_spectra_workspace_bytes(2, 1, 8) == 0
    assert lib.hitb200_spectra_fields(None, p, p, 1, 8, 8, 0, p, p, 64, None) == _lib.ERR_INVALID
    assert lib.hitb200_spectra_fields(p, p, p, 0, 8, 8, 0, p, p, 64, None) == _lib.ERR_INVALID
    # workspace too small for the call
    assert lib.hitb200_spectra_fields(p, p, p, 1, 64, 64, 0, p, p, 64, None) == _lib.ERR_INVALID
    assert lib.hitb200_spectra_shells(p, 1, 64, 64, 0.0, 0.1, p, p, p, 1 << 30, None) == _lib.ERR_INVALID
    st = lib.hitb200_spectra_shells(p, 1, 4100, 4100, 0.1, 0.1, p, p, p, 1 << 40, None)
    assert st == _lib.ERR_UNSUPPORTED
    assert "1025" in lib.hitb200_status_string(st).decode()


def test_mirror_constructor_and_selection_errors(tmp_path):
    from hit_solver_b200.postprocess import HIT2DSpectra

    with pytest.raises(ValueError):
        HIT2DSpectra(tmp_path, fluctuation_type="mass")
    with pytest.raises(ValueError):
        HIT2DSpectra(tmp_path, stride=0)
    with pytest.raises(FileNotFoundError):
        HIT2DSpectra(tmp_path).compute()
    np.savez(tmp_path / "hit2d_step0000000.npz", time=1.0)
    with pytest.raises(ValueError):
        HIT2DSpectra(tmp_path, end_time=0.5).compute()
    with pytest.raises(RuntimeError):
        HIT2DSpectra(tmp_path).save()
