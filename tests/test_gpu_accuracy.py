"""Accuracy of the FP32-bulk form over a long production HIT run.

The 512^2 production forced HIT (OU forcing on shell 3..5 with Mach control,
viscosity, hyperviscosity every 5 steps, drag, cooling) runs 1000 steps in the
plain FP64 form and in the FP32-bulk form with the same device forcing noise.
The FP64 form is itself held to the oracle step by step by the parity tests.
Kinetic energy, enstrophy (mean vorticity^2, spectral as in the reference's
diagnostics), turbulent Mach number and the injected forcing power of the
FP32-bulk run must stay within 1e-4 relative of the FP64 run.
"""

import pytest
import torch

from hit_solver_b200 import _lib
from hit_solver_b200.hit2d import HITSolver, compute_diagnostics
from hit_solver_b200.serving import hit_request_config

RTOL = 1e-4
STEPS = 1000


def _run(precision):
    s = HITSolver(hit_request_config(512, 1234, 0.25, STEPS, precision))
    s.advance(STEPS)
    torch.cuda.synchronize()
    sc = s.plan.scalars()
    assert int(sc[_lib.S_STEP]) == STEPS and int(sc[_lib.S_STATUS]) == 0
    d = compute_diagnostics(s.q, s.equation, s.domain)
    return d, sc


@pytest.mark.gpu
def test_fp32_bulk_tracks_fp64_over_1000_steps():
    d64, s64 = _run("fp64")
    d32, s32 = _run("fp32-bulk")
    for key in ("kinetic_energy", "turbulent_mach", "rms_velocity"):
        assert abs(d32[key] - d64[key]) <= RTOL * abs(d64[key]), (key, d32[key], d64[key])
    ens32, ens64 = d32["vorticity_rms"] ** 2, d64["vorticity_rms"] ** 2
    assert abs(ens32 - ens64) <= RTOL * ens64, ("enstrophy", ens32, ens64)
    p32, p64 = s32[_lib.S_F_INJECTED], s64[_lib.S_F_INJECTED]
    assert abs(p32 - p64) <= RTOL * abs(p64), ("forcing power", p32, p64)
    assert abs(s32[_lib.S_TIME] - s64[_lib.S_TIME]) <= RTOL * s64[_lib.S_TIME]


@pytest.mark.gpu
def test_fp32_bulk_long_riemann_stays_finite():
    # Riemann configuration 3 at 896^2 with x0 = y0 = 0.58287: in the FP32-bulk
    # form a WENO weight denominator (eps + IS_0)^2 once cancelled to below
    # FP32 range near step 1990 and turned the state non-finite; the floored
    # denominator keeps the run finite to tfinal, close to the FP64 minimum
    # density (0.13659).
    from hit_solver_b200 import serving

    req = serving.Request(0, "riemann3", 896, split=0.5828655255129153)
    s = serving.make_solver(req, "fp32-bulk")
    s.advance(s.n_steps)
    sc = s.plan.scalars()
    assert int(sc[_lib.S_STEP]) == s.n_steps == 2350
    assert int(sc[_lib.S_STATUS]) == 0
    assert bool(torch.isfinite(s.q).all())
    assert abs(float(s.q[0].min()) - 0.13659) < 2e-3
