"""Output-file compatibility with the reference's own writers.

``tests/golden/formats_*.npz`` hold every file that the reference wrote for
a short 24^2 HIT run (``run_simulation``: config.json, diagnostic_history.npz
and the snapshots, OOP/hit2d.py:551-694, 764-918) and a 24^2 Riemann
configuration-3 run (``run_riemann`` + ``save_run_outputs`` without the
figure, OOP/problems/riemann_config3.py:486-519, 681-809), flattened as
``<file>::<key>`` arrays (``tests/golden/make_golden.py``).  The same runs
through the b200 mirror must write the same files with the same keys,
dtypes and shapes, and the same values within the FP64 tolerance of the
parity tests; the configuration JSON may add the mirror's own fields.
"""

import json
import tempfile
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
# the FP64 tolerance of the parity tests for states after short runs (relative
# to the largest magnitude of the compared array); derived fields (vorticity)
# carry the state's roundoff differences divided by the mesh width
RTOL = 1e-8


def _collect(tmp: Path) -> dict:
    out = {}
    for path in sorted(tmp.rglob("*")):
        if path.is_dir():
            continue
        rel = path.relative_to(tmp).as_posix()
        if path.suffix == ".npz":
            with np.load(path, allow_pickle=False) as d:
                for k in d.files:
                    out[f"{rel}::{k}"] = d[k]
        elif path.suffix == ".json":
            out[rel] = np.asarray(path.read_text())
    return out


# the mirror's configuration adds these fields and runs on its own backend
_MIRROR_ONLY = {"precision", "forcing_noise", "max_steps", "initial_condition"}
_DIFFERS = {"backend", "output_dir"}


def _same_json(got: str, want: str):
    g, w = json.loads(got), json.loads(want)
    assert set(w) <= set(g), set(w) - set(g)
    assert set(g) - set(w) <= _MIRROR_ONLY, set(g) - set(w)
    for k, v in w.items():
        if k in _DIFFERS:
            continue
        if isinstance(v, float) and isinstance(g[k], float):
            assert abs(g[k] - v) <= RTOL * max(abs(v), 1e-300) or (np.isnan(v) and np.isnan(g[k])), k
        else:
            assert g[k] == v, (k, g[k], v)


def _compare(got: dict, want: dict, scale_of=None):
    assert sorted(got) == sorted(want)
    for key, w in want.items():
        g = got[key]
        # strings (JSON text) may differ in length; every other dtype must match
        same_type = g.dtype.kind == "U" if w.dtype.kind == "U" else g.dtype == w.dtype
        assert same_type and g.shape == w.shape, (key, g.dtype, w.dtype, g.shape, w.shape)
        if w.dtype.kind == "U":
            if key.endswith(".json") or key.endswith("_json"):
                _same_json(str(g), str(w))
            else:
                assert str(g) == str(w), key
            continue
        if w.dtype.kind in "biu":
            np.testing.assert_array_equal(g, w, err_msg=key)
            continue
        scale = max(float(np.nanmax(np.abs(w))) if w.size else 0.0, scale_of(key) if scale_of else 0.0)
        np.testing.assert_allclose(g, w, rtol=0, atol=RTOL * max(scale, 1e-300), err_msg=key)


@pytest.mark.gpu
def test_hit_run_files_match_reference():
    from hit_solver_b200 import hit2d

    want = dict(np.load(GOLD / "formats_hit_24.npz"))
    with tempfile.TemporaryDirectory() as t:
        cfg = hit2d.HIT2DConfig(nx=24, ny=24, tfinal=0.006, cfl=0.05, target_mach=0.25,
                                initial_kmin=3, initial_kmax=5, forcing_kmin=3.0,
                                forcing_kmax=5.0, forcing_correlation_time=0.5,
                                mach_control=True, mach_control_target=0.25, viscosity=7.5e-4,
                                large_scale_drag=0.1, cooling_time=5.0, hyperviscosity_mn=0.002,
                                diagnostics_every=2, snapshot_every=3, output_dir=Path(t),
                                precision="fp64")
        hit2d.run_simulation(cfg)
        got = _collect(Path(t))

    # divergence values are roundoff of a solenoidal field: compare them on the
    # scale of the vorticity of the same snapshot or history
    def scale_of(key):
        if key.endswith("::divergence"):
            return float(np.max(np.abs(want[key.replace("divergence", "vorticity")])))
        if key.endswith("::divergence_rms"):
            return float(np.max(want[key.replace("divergence_rms", "vorticity_rms")]))
        if key.endswith(("::A_K", "::C_uv", "::A_F", "::Fxy", "::mass_error")):
            return 1.0
        return 0.0

    _compare(got, want, scale_of)


@pytest.mark.gpu
def test_riemann_run_files_match_reference():
    from hit_solver_b200.problems import riemann as R

    want = dict(np.load(GOLD / "formats_riemann_24.npz"))
    cfg = R.RiemannConfig3(nx=24, ny=24, tfinal=0.02, shear_threshold=None, progress_every=10 ** 6)
    q, diag = R.run_riemann(cfg)
    with tempfile.TemporaryDirectory() as t:
        R.save_run_outputs(q, cfg, diag, Path(t), run_id="fixture")
        got = _collect(Path(t))
    _compare(got, want)


def test_mirror_reads_the_reference_riemann_file():
    """load_riemann_npz of the mirror on a file written by the reference."""
    from hit_solver_b200.problems import riemann as R

    want = dict(np.load(GOLD / "formats_riemann_24.npz"))
    members = {k.split("::", 1)[1]: v for k, v in want.items() if "::" in k}
    with tempfile.TemporaryDirectory() as t:
        path = Path(t) / "ref_final.npz"
        np.savez_compressed(path, **members)
        data, cfg = R.load_riemann_npz(path)
        assert cfg.nx == 24 and cfg.tfinal == 0.02 and cfg.shear_threshold is None
        assert int(data["steps"]) == int(members["steps"])
        np.testing.assert_array_equal(data["q"], members["q"])
