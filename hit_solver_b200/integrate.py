"""The reference-side integration of the b200 backend, applied to a copy.

``patch_tree(reference_root, destination)`` copies a HIT_Solver source tree
and adds the ``b200`` branches a maintainer adds by hand (the patch shown in
INTEGRATION.md):

* ``OOP/parallel/backend.py`` ``select_array_module`` returns torch for
  ``"b200"`` after loading the native library (``RuntimeError`` without a
  CUDA device, as the reference raises for a missing backend);
* ``OOP/hit2d.py`` ``run_simulation`` and
  ``OOP/problems/riemann_config3.py`` ``run_riemann`` hand a ``b200``
  configuration to the mirror's drivers;
* the ``--backend`` choices of ``OOP/hit2d.py`` and
  ``scripts/run_riemann_config*.py`` gain ``"b200"``.

Each edit is anchored on the reference's own definition lines and fails
loudly if an anchor is missing, so that a change of the reference is noticed.

    python -m hit_solver_b200.integrate <reference-root> <destination>
"""

from __future__ import annotations

import shutil
import sys
from pathlib import Path

_BACKEND = """    if backend == "b200":
        import torch

        import hit_solver_b200

        hit_solver_b200.core.require_cuda()
        return torch
"""
_RUN_HIT = """    if config.backend == "b200":
        from hit_solver_b200.hit2d import run_simulation as _run_b200

        return _run_b200(config)
"""
_RUN_RIEMANN = """    if config.backend == "b200":
        from hit_solver_b200.problems.riemann import run_riemann as _run_b200

        return _run_b200(config)
"""
_CHOICES_OLD = 'choices=("auto", "numpy", "cupy")'
_CHOICES_NEW = 'choices=("auto", "numpy", "cupy", "b200")'


def _insert_after(path: Path, anchor: str, text: str) -> None:
    lines = path.read_text().splitlines(keepends=True)
    for i, line in enumerate(lines):
        if line.startswith(anchor):
            lines.insert(i + 1, text)
            path.write_text("".join(lines))
            return
    raise RuntimeError(f"{path}: anchor {anchor!r} not found")


def _extend_choices(path: Path) -> None:
    src = path.read_text()
    if _CHOICES_OLD not in src:
        raise RuntimeError(f"{path}: --backend choices not found")
    path.write_text(src.replace(_CHOICES_OLD, _CHOICES_NEW))


def patch_tree(reference_root, destination) -> list[str]:
    """Copy the tree and apply the b200 branches; returns the edited files."""
    src, dst = Path(reference_root), Path(destination)
    shutil.copytree(src, dst, ignore=shutil.ignore_patterns("results", "__pycache__", ".git"))
    dst.chmod(0o755)
    for p in dst.rglob("*"):
        p.chmod(0o755 if p.is_dir() else 0o644)
    edited = []
    f = dst / "OOP" / "parallel" / "backend.py"
    _insert_after(f, "def select_array_module(backend: str):", _BACKEND)
    edited.append(f)
    f = dst / "OOP" / "hit2d.py"
    _insert_after(f, "def run_simulation(config: HIT2DConfig)", _RUN_HIT)
    edited.append(f)
    f = dst / "OOP" / "problems" / "riemann_config3.py"
    _insert_after(f, "def run_riemann(config: RiemannConfig3):", _RUN_RIEMANN)
    edited.append(f)
    for script in sorted((dst / "scripts").glob("run_riemann_config*.py")):
        _extend_choices(script)
        edited.append(script)
    src_hit = (dst / "OOP" / "hit2d.py").read_text()
    start = src_hit.index('"--backend"')
    seg = src_hit[start:start + 200]
    if "choices" in seg:
        _extend_choices(dst / "OOP" / "hit2d.py")
    return [str(p.relative_to(dst)) for p in edited]


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit("usage: python -m hit_solver_b200.integrate <reference-root> <destination>")
    for name in patch_tree(sys.argv[1], sys.argv[2]):
        print("patched", name)
