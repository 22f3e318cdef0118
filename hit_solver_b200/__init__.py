"""B200-native backend for the HIT_Solver hot path.

The right-hand side and SSP-RK3 step of the reference's 2-D compressible
solver (hybrid compact-FD / WENO7 flux, shock sensor, hyperviscosity,
viscous and thermal terms, OU forcing with Mach control, drag, cooling and
the reductions that drive them) as hand-written sm_100a CUDA kernels behind a
C ABI (``include/hitb200.h``, ``libhitb200.so``).  The Python modules mirror
the reference's classes and drivers with ``backend="b200"``; arrays are torch
CUDA tensors.

Submodules are imported lazily so that ``import hit_solver_b200`` works on a
machine without a GPU (the C library still loads; calls need a device).
"""

from __future__ import annotations

__all__ = ["build", "core", "hit2d", "problems", "spatial_operator", "equations", "forcing",
           "time_operator", "domain", "backend", "batch", "serving", "postprocess"]


def __getattr__(name):
    import importlib

    if name in __all__:
        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(name)
