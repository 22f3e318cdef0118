"""Four-quadrant 2-D Riemann problems on the B200 backend
(OOP/problems/__init__.py)."""

from .riemann import (RiemannConfig3, RiemannConfig3Offset08, RiemannConfig6, RiemannDiagnostics,
                      run_riemann, run_riemann_config3, run_riemann_config3_08,
                      run_riemann_config6)

__all__ = ["RiemannConfig3", "RiemannConfig3Offset08", "RiemannConfig6", "RiemannDiagnostics",
           "run_riemann", "run_riemann_config3", "run_riemann_config3_08", "run_riemann_config6"]
