"""The x sweep's stage epilogue takes two nodes per thread with 16-byte
(FP64) and 8-byte (FP32) vector accesses when the row length is even and
every state pointer it touches is 16-byte aligned, one node per thread
otherwise.  The two forms must give the same bits: a solve whose state
tensor starts 8 bytes past an aligned address (a view at element 1 of a
larger buffer) runs the scalar form and is compared with the same solve on
an aligned tensor."""

import pytest
import torch


def _unaligned_like(q):
    buf = torch.empty(q.numel() + 1, dtype=q.dtype, device=q.device)
    v = buf[1:].view_as(q)
    v.copy_(q)
    assert v.data_ptr() % 16 == 8
    return v


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32-bulk"])
def test_hit_steps_identical_on_unaligned_state(precision):
    from hit_solver_b200.hit2d import HIT2DConfig, HITSolver

    cfg = HIT2DConfig(nx=64, ny=48, tfinal=1e9, cfl=0.05, target_mach=0.25, initial_kmin=3,
                      initial_kmax=5, forcing_kmin=3.0, forcing_kmax=5.0,
                      forcing_correlation_time=0.5, mach_control=True, viscosity=7.5e-4,
                      large_scale_drag=0.1, cooling_time=5.0, hyperviscosity_mn=0.002,
                      hyperviscosity_interval=2, forcing_noise="device", precision=precision)
    a, b = HITSolver(cfg), HITSolver(cfg)
    b.q = _unaligned_like(b.q)
    assert torch.equal(a.q, b.q)
    a.advance(5)
    b.advance(5)
    torch.cuda.synchronize()
    assert torch.equal(a.q, b.q)
    assert a.scalars() == b.scalars()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32-bulk"])
def test_riemann_steps_identical_on_unaligned_state(precision):
    from hit_solver_b200.problems.riemann import RiemannConfig3, RiemannSolver

    cfg = RiemannConfig3(nx=96, ny=64, tfinal=0.05, backend="b200", precision=precision,
                         progress_every=10**9)
    a, b = RiemannSolver(cfg), RiemannSolver(cfg)
    b.q = _unaligned_like(b.q)
    a.advance(6)
    b.advance(6)
    torch.cuda.synchronize()
    assert torch.equal(a.q, b.q)
