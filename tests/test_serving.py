"""Continuous-batching request loop (hit_solver_b200.serving).

The GPU test runs a small mixed stream (Riemann configurations 3 and 6 and
forced HIT, uneven grid sizes, staggered arrivals, a memory budget that
forces queueing) and checks that every request's final state equals the same
request run alone through the plain single-solve path.  The stated tolerance
is exact equality: each solve's kernels and reductions touch only its own
data in a fixed order, so batching must not change a single bit.
"""

import pytest
import torch

from hit_solver_b200 import serving


def test_poisson_stream_is_seeded_and_in_range():
    a = serving.poisson_requests(40, 20.0, seed=3)
    b = serving.poisson_requests(40, 20.0, seed=3)
    assert [(r.kind, r.n, r.arrival, r.split, r.seed, r.mach) for r in a] == \
           [(r.kind, r.n, r.arrival, r.split, r.seed, r.mach) for r in b]
    arr = [r.arrival for r in a]
    assert arr == sorted(arr) and arr[0] > 0.0
    for r in a:
        assert r.kind in serving.KINDS
        if r.kind == "hit":
            assert 128 <= r.n <= 512 and 0.1 <= r.mach <= 0.4 and r.steps == 200
        else:
            assert 256 <= r.n <= 1024 and 0.3 <= r.split <= 0.8
        assert r.n % 64 == 0


def test_footprint_grows_with_grid():
    small = serving.footprint(serving.Request(0, "riemann3", 64), "fp32-bulk")
    large = serving.footprint(serving.Request(1, "riemann3", 128), "fp32-bulk")
    hit = serving.footprint(serving.Request(2, "hit", 64), "fp32-bulk")
    assert 0 < small < large
    assert hit > 4 * 64 * 64 * 8


def test_unknown_kind_rejected():
    with pytest.raises(ValueError):
        serving.make_solver(serving.Request(0, "sod", 32), "fp32-bulk")


@pytest.mark.gpu
def test_mixed_stream_matches_solo_runs():
    reqs = [
        serving.Request(0, "riemann3", 64, 0.00, split=0.5),
        serving.Request(1, "hit", 48, 0.00, seed=11, mach=0.2, steps=23),
        serving.Request(2, "riemann6", 40, 0.01, split=0.4),
        serving.Request(3, "hit", 64, 0.02, seed=5, mach=0.3, steps=37),
        serving.Request(4, "riemann3", 32, 0.03, split=0.7),
    ]
    # room for about three of them at a time: later arrivals queue for memory
    budget = sum(sorted(serving.footprint(r, "fp32-bulk") for r in reqs)[-3:])
    server = serving.SolveServer("fp32-bulk", hbm_budget=budget, steps_per_round=8,
                                 keep_states=True)
    results = server.serve(reqs)
    assert sorted(r.rid for r in results) == [0, 1, 2, 3, 4]
    assert server.stats["rounds"] > 1 and server.stats["p99_s"] >= server.stats["p50_s"] > 0.0
    for res in results:
        req = reqs[res.rid]
        assert res.status == 0
        if req.kind == "hit":
            assert res.steps == req.steps
        solo = serving.run_alone(req, "fp32-bulk")
        assert torch.equal(res.state, solo), f"request {res.rid} differs from its solo run"


def test_member_error_mapping():
    from hit_solver_b200 import _lib

    assert serving.member_error("hit", 0) is None
    assert serving.member_error("riemann3", 0) is None
    assert serving.member_error("hit", _lib.ST_NONFINITE)[0] == "FloatingPointError"
    assert serving.member_error("hit", _lib.ST_BARRIER)[0] == "RuntimeError"
    # the reference validates positivity only in its Riemann loop
    assert serving.member_error("hit", _lib.ST_NONPOS_RHO) is None
    assert serving.member_error("riemann6", _lib.ST_NONPOS_P)[0] == "FloatingPointError"


@pytest.mark.gpu
def test_nan_request_is_evicted_and_others_unaffected():
    """A request whose initial state holds a NaN (injected on the host) is
    evicted at the end of its first round with the reference's
    FloatingPointError, while its batch companions run to their end and
    equal their solo runs bit for bit (OOP/hit2d.py:716-717;
    OOP/problems/riemann_config3.py:442-452)."""
    good = serving.make_solver(serving.Request(9, "riemann3", 48, split=0.55), "fp32-bulk")
    bad_state = good.q.clone()
    bad_state[2, 20, 31] = float("nan")
    reqs = [
        serving.Request(0, "hit", 48, 0.0, seed=3, mach=0.25, steps=30),
        serving.Request(1, "riemann3", 48, 0.0, split=0.55, initial_state=bad_state),
        serving.Request(2, "riemann6", 40, 0.0, split=0.45),
    ]
    server = serving.SolveServer("fp32-bulk", steps_per_round=8, keep_states=True)
    results = {r.rid: r for r in server.serve(reqs)}
    assert set(results) == {0, 1, 2}
    bad = results[1]
    assert bad.error_type == "FloatingPointError" and "NaN" in bad.error
    assert bad.steps <= 8  # evicted at the first round boundary
    assert server.stats["failed"] == 1
    for rid in (0, 2):
        res = results[rid]
        assert res.error is None and res.status == 0
        assert torch.equal(res.state, serving.run_alone(reqs[rid], "fp32-bulk"))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["hit", "riemann3"])
def test_checkpoint_restore_resumes_bit_for_bit(kind):
    """q plus the plan's scalar block (time, step, controller and forcing
    state, OU potential; the device noise is keyed by seed and step) resume a
    solve exactly: 7 + 9 steps through a checkpoint equal 16 straight steps."""
    req = serving.Request(0, kind, 64, split=0.6, seed=8, mach=0.3, steps=10 ** 6)
    straight = serving.make_solver(req, "fp32-bulk")
    straight.advance(16)
    first = serving.make_solver(req, "fp32-bulk")
    first.advance(7)
    ck = first.checkpoint()
    del first
    resumed = serving.make_solver(req, "fp32-bulk")
    resumed.restore(ck)
    resumed.advance(9)
    torch.cuda.synchronize()
    assert torch.equal(resumed.q, straight.q)
    assert resumed.plan.scalars() == straight.plan.scalars()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["run", "step"])
def test_mixed_line_classes_match_solo_runs(mode):
    """Members whose grid lines fall in different nodes-per-thread classes of
    the sweeps (up to 128, 256, 512 and 1024 nodes; one member with x and y
    lines in different classes) keep the bits of their solo runs: a batch
    launches each class's sweeps separately, with the class a member has
    alone."""
    from hit_solver_b200.batch import Batch
    from hit_solver_b200.problems.riemann import RiemannConfig3, RiemannSolver

    def members():
        return [serving.make_solver(serving.Request(0, "hit", 64, seed=2, mach=0.25, steps=10 ** 6),
                                    "fp32-bulk"),
                serving.make_solver(serving.Request(1, "riemann3", 200, split=0.45), "fp32-bulk"),
                RiemannSolver(RiemannConfig3(nx=320, ny=96, precision="fp32-bulk")),
                serving.make_solver(serving.Request(3, "riemann6", 640, split=0.6), "fp32-bulk")]

    sv = members()
    b = Batch.from_plans([s.plan for s in sv], [s.q for s in sv])
    if mode == "run":
        b.run(5)
    else:
        for _ in range(5):
            b.step()
    torch.cuda.synchronize()
    got = [s.q.clone() for s in sv]
    b.close()
    for i, ref in enumerate(members()):
        ref.advance(5)
        torch.cuda.synchronize()
        assert torch.equal(got[i], ref.q), f"member {i} differs from its solo run"
