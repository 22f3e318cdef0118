"""Failure detection of the fused prepass + sensor's grid barrier.

The cooperative sensor launch meets at a grid barrier whose wait is bounded
(the global timer; 2 s by default).  A host-side test hook makes the barrier
wait for one CTA more than the launch has, so that every wait runs out after
1 ms: each CTA withdraws its arrival, the step reports HITB200_ST_BARRIER
(the run loops raise RuntimeError) and the GPU stays usable: a fresh solve
then runs the fused step normally and equals the two-kernel path bit for
bit.  The same hook lengthens the waits of the persistent stage kernel
(each item's wait for its solve's previous phase) by one arrival: the first
wait runs out, the launch's other waits end at once, every member reports
HITB200_ST_BARRIER, and the next batch runs normally.  No GPU fault, trap or
endless wait is involved.
"""

import pytest
import torch

from hit_solver_b200 import _lib, serving
from hit_solver_b200.batch import Batch


def test_barrier_test_hook_rejects_bad_arguments():
    lib = _lib.load()
    assert lib.hitb200_set_barrier_test(2, 1e-3) == _lib.ERR_INVALID
    assert lib.hitb200_set_barrier_test(-1, 1e-3) == _lib.ERR_INVALID
    assert lib.hitb200_set_barrier_test(1, 0.0) == _lib.ERR_INVALID
    assert lib.hitb200_set_barrier_test(1, 60.0) == _lib.ERR_INVALID


@pytest.mark.gpu
def test_fused_barrier_timeout_reports_and_recovers():
    lib = _lib.load()
    req = serving.Request(0, "riemann3", 64, split=0.5)
    s = serving.make_solver(req, "fp32-bulk")
    s.plan.set_tuning([0, 0, 0, 1, 0, 0])
    _lib.check(lib.hitb200_set_barrier_test(1, 1e-3))
    try:
        s.advance(1)
        torch.cuda.synchronize()
        bits = int(s.plan.scalars()[_lib.S_STATUS])
    finally:
        _lib.check(lib.hitb200_set_barrier_test(0, 2.0))
    assert bits & _lib.ST_BARRIER
    with pytest.raises(RuntimeError):
        _lib.check_step_status(bits, "Riemann state")
    # the device and the library recover: fused and two-kernel steps agree
    fused = serving.make_solver(req, "fp32-bulk")
    fused.plan.set_tuning([0, 0, 0, 1, 0, 0])
    plain = serving.make_solver(req, "fp32-bulk")
    fused.advance(4)
    plain.advance(4)
    torch.cuda.synchronize()
    assert int(fused.plan.scalars()[_lib.S_STATUS]) == 0
    assert torch.equal(fused.q, plain.q)


def _small_batch_members():
    return [serving.make_solver(serving.Request(0, "hit", 64, seed=5, mach=0.2, steps=10 ** 6), "fp32-bulk"),
            serving.make_solver(serving.Request(1, "riemann3", 48, split=0.4), "fp32-bulk")]


@pytest.mark.gpu
def test_persistent_stage_wait_timeout_reports_and_recovers():
    lib = _lib.load()
    sv = _small_batch_members()
    b = Batch.from_plans([s.plan for s in sv], [s.q for s in sv])
    b.set_tuning([1, 1, 1, 0, 0, 1])
    assert b.tuning[_lib.TUNE_PERSISTENT] == 1
    _lib.check(lib.hitb200_set_barrier_test(1, 1e-3))
    try:
        b.step()
        torch.cuda.synchronize()
    finally:
        _lib.check(lib.hitb200_set_barrier_test(0, 2.0))
    # a wait that ran out is reported by the member's next prepass
    b.step()
    torch.cuda.synchronize()
    bits = [int(s.plan.scalars()[_lib.S_STATUS]) for s in sv]
    b.close()
    for x in bits:
        assert x & _lib.ST_BARRIER
    with pytest.raises(RuntimeError):
        _lib.check_step_status(bits[0], "HIT state")
    # the device, the queue and the counters recover: persistent and
    # per-phase batches agree bit for bit
    finals = []
    for persist in (1, 0):
        sv = _small_batch_members()
        b = Batch.from_plans([s.plan for s in sv], [s.q for s in sv])
        b.set_tuning([1, 1, 1, 0, 0, persist])
        b.run(3)
        torch.cuda.synchronize()
        assert all(int(s.plan.scalars()[_lib.S_STATUS]) == 0 for s in sv)
        finals.append([s.q.clone() for s in sv])
        b.close()
    for a, c in zip(*finals):
        assert torch.equal(a, c)
