"""The reference-side patch of INTEGRATION.md, applied to a copy of the
reference (hit_solver_b200.integrate.patch_tree): ``--backend b200`` reaches
the mirror's drivers.  Runs on the CPU with the native drivers stubbed; it
needs the reference's source tree, named by the HIT_SOLVER_REFERENCE
environment variable, and is skipped without it."""

import importlib
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

REF = os.environ.get("HIT_SOLVER_REFERENCE")
ROOT = Path(__file__).resolve().parent.parent
STUBS = Path(__file__).resolve().parent / "golden" / "_stubs"

pytestmark = pytest.mark.skipif(not REF or not Path(REF, "OOP").is_dir(),
                                reason="HIT_SOLVER_REFERENCE does not name a reference tree")


def test_patch_dispatches_b200_to_the_mirror(tmp_path):
    from hit_solver_b200.integrate import patch_tree

    dst = tmp_path / "ref"
    edited = patch_tree(REF, dst)
    assert "OOP/parallel/backend.py" in edited and "OOP/hit2d.py" in edited
    assert "OOP/problems/riemann_config3.py" in edited
    # a fresh interpreter imports the patched reference, with the mirror's
    # native drivers replaced by recorders (no GPU on this machine)
    probe = textwrap.dedent(f"""
        import sys
        sys.path[:0] = [{str(STUBS)!r}, {str(dst)!r}, {str(ROOT)!r}]
        import hit_solver_b200.hit2d as H
        import hit_solver_b200.problems.riemann as RB
        import hit_solver_b200.core as C
        calls = []
        H.run_simulation = lambda cfg: calls.append(("hit", type(H.as_config(cfg)).__module__, cfg.nx)) or "hit-ok"
        RB.run_riemann = lambda cfg: calls.append(("riemann", type(RB.as_config(cfg)).__name__, cfg.nx)) or "riemann-ok"
        C.require_cuda = lambda: None
        from OOP import hit2d
        from OOP.parallel.backend import select_array_module
        from OOP.problems import riemann_config3 as rc3
        from OOP.problems.riemann_config6 import RiemannConfig6
        assert select_array_module("b200").__name__ == "torch"
        assert hit2d.run_simulation(hit2d.HIT2DConfig(nx=16, ny=16, backend="b200")) == "hit-ok"
        assert rc3.run_riemann(RiemannConfig6(nx=24, ny=24, backend="b200")) == "riemann-ok"
        try:
            select_array_module("bogus")
        except ValueError:
            pass
        else:
            raise SystemExit("unknown backend not rejected")
        print(calls)
        assert calls == [("hit", "hit_solver_b200.hit2d", 16), ("riemann", "RiemannConfig6", 24)]
    """)
    res = subprocess.run([sys.executable, "-c", probe], capture_output=True, text=True, cwd=tmp_path)
    assert res.returncode == 0, res.stdout + res.stderr
