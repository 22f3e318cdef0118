"""Kernel variants and the autotuner (hit_solver_b200.autotune).

The variants differ only in register budgets and CTAs per SM, so the state
after any number of steps must be bit-identical whichever variants run; the
tuner must return one valid choice per kernel family and apply it.
"""

import pytest
import torch

from hit_solver_b200 import _lib, autotune, serving
from hit_solver_b200.batch import Batch


def _mixed(n_hit=48, n_riem=40):
    hit = serving.make_solver(serving.Request(0, "hit", n_hit, seed=3, mach=0.3, steps=10 ** 6),
                              "fp32-bulk")
    riem = serving.make_solver(serving.Request(1, "riemann3", n_riem, split=0.45), "fp32-bulk")
    return [hit, riem]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32-bulk", "fp64"])
def test_variants_give_identical_states(precision):
    finals = []
    for knobs in ([0, 0, 0, 0, 0, 0], [1, 1, 1, 0, 1, 0], [1, 0, 1, 0, 0, 1], [0, 1, 0, 0, 1, 1]):
        sv = [serving.make_solver(serving.Request(0, "hit", 48, seed=3, mach=0.3, steps=10 ** 6), precision),
              serving.make_solver(serving.Request(1, "riemann3", 40, split=0.45), precision)]
        b = Batch.from_plans([s.plan for s in sv], [s.q for s in sv])
        b.set_tuning(knobs)
        # the persistent stage form is an FP32-bulk batch form
        want = list(knobs)
        if precision == "fp64":
            want[_lib.TUNE_PERSISTENT] = 0
        assert b.tuning == want
        b.run(7)
        torch.cuda.synchronize()
        finals.append([s.q.clone() for s in sv])
        b.close()
    for other in finals[1:]:
        for a, c in zip(finals[0], other):
            assert torch.equal(a, c)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,n", [("riemann6", 64), ("riemann3", 96), ("hit", 64)])
def test_single_plan_variants_identical(kind, n):
    # includes the fused prepass + sensor (knob 3), whose grid-barrier path
    # must reproduce the two-kernel path bit for bit, and the y sweep's other
    # panel width (knob 4)
    out = []
    for knobs in ([0, 0, 0, 0, 0, 0], [1, 1, 1, 0, 0, 0], [0, 0, 0, 1, 1, 0], [1, 1, 1, 1, 1, 0],
                  [0, 1, 0, 0, 1, 0]):
        s = serving.make_solver(serving.Request(0, kind, n, split=0.5, seed=4, steps=10 ** 6),
                                "fp32-bulk")
        s.plan.set_tuning(knobs)
        assert s.plan.tuning == knobs
        s.advance(6)
        torch.cuda.synchronize()
        assert int(s.plan.scalars()[_lib.S_STATUS]) == 0
        out.append(s.q.clone())
    for o in out[1:]:
        assert torch.equal(out[0], o)


@pytest.mark.gpu
def test_autotune_batch_and_plan():
    autotune.clear_cache()
    sv = _mixed()
    b = Batch.from_plans([s.plan for s in sv], [s.q for s in sv])
    before = [s.q.clone() for s in sv]
    knobs = b.autotune(trials=1)
    assert len(knobs) == _lib.TUNE_COUNT and set(knobs) <= {0, 1}
    assert b.tuning == knobs
    # tuning ran on copies: the batch's own states are untouched
    for a, c in zip(before, [s.q for s in sv]):
        assert torch.equal(a, c)
    # cached: same answer without timing again
    assert autotune.tune_batch(b) == knobs
    b.close()
    s = serving.make_solver(serving.Request(2, "riemann3", 64, split=0.5), "fp32-bulk")
    k2 = autotune.tune_plan(s.plan, s.q, trials=1)
    assert s.plan.tuning == k2


@pytest.mark.gpu
def test_autotune_choice_read_back_from_disk(tmp_path, monkeypatch):
    """A later process (here: an emptied in-memory cache) takes the measured
    choice from the disk cache without timing again."""
    monkeypatch.setenv("HITB200_TUNE_CACHE", str(tmp_path / "tuning.json"))
    autotune.clear_cache()
    s = serving.make_solver(serving.Request(3, "riemann6", 96, split=0.4), "fp32-bulk")
    k = autotune.tune_plan(s.plan, s.q, trials=1)
    autotune.clear_cache()

    def no_timing(*a, **kw):
        raise AssertionError("tuned again instead of reading the disk cache")

    monkeypatch.setattr(autotune, "_choose", no_timing)
    s.plan.set_tuning([-1] * _lib.TUNE_COUNT)
    assert autotune.tune_plan(s.plan, s.q) == k
    assert s.plan.tuning == k
    autotune.clear_cache()


@pytest.mark.gpu
def test_tuning_knob_validation():
    s = serving.make_solver(serving.Request(0, "riemann3", 32), "fp32-bulk")
    with pytest.raises(ValueError):
        s.plan.set_tuning([2, 0, 0])
    with pytest.raises(ValueError):
        s.plan.set_tuning([0] * (_lib.TUNE_COUNT + 1))
    s.plan.set_tuning([-1] * _lib.TUNE_COUNT)  # back to the launch-size default
    assert set(s.plan.tuning) <= {0, 1}


def _uneven_members():
    """FP32-bulk solves of uneven, non-square grids, some with line lengths
    that are not multiples of 4 (the last x group / y panel of a member holds
    fewer than 4 lines): production HIT (viscous, forced, drag, cooling,
    hyperviscosity every 5 steps) and Riemann configurations 3 and 6
    (outflow edges, guard cells, hyperviscosity every step); all lines of at
    most 128 nodes (one nodes-per-thread class, as the persistent form
    requires)."""
    from hit_solver_b200.hit2d import HITSolver
    from hit_solver_b200.problems.riemann import RiemannConfig3, RiemannConfig6, RiemannSolver

    import dataclasses

    out = []
    for i, (nx, ny) in enumerate([(64, 48), (96, 80), (37, 61), (128, 128)]):
        # the 37 x 61 solve stops after 3 steps: a finished member's items
        # must still count for its phase counters
        steps = 3 if i == 2 else 10 ** 6
        cfg = serving.hit_request_config(64, 10 + i, 0.15 + 0.05 * i, steps, "fp32-bulk")
        out.append(HITSolver(dataclasses.replace(cfg, nx=nx, ny=ny)))
    out.append(RiemannSolver(RiemannConfig3(nx=37, ny=29, x_split=0.45, y_split=0.55, precision="fp32-bulk")))
    out.append(RiemannSolver(RiemannConfig6(nx=50, ny=66, precision="fp32-bulk")))
    out.append(RiemannSolver(RiemannConfig3(nx=120, ny=100, precision="fp32-bulk")))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("steps", [1, 6])
def test_persistent_stage_matches_per_phase_launches(steps):
    """One persistent launch per RK3 stage (knob 5) against one launch per
    phase: the same states bit for bit after every member's first step
    (whose first stage has no prepass items) and after several steps,
    replayed from the two-branch graph and stepped plainly."""
    finals = {}
    for persist in (0, 1):
        for mode in ("run", "step"):
            sv = _uneven_members()
            b = Batch.from_plans([s.plan for s in sv], [s.q for s in sv])
            knobs = [1, 1, 1, 0, 0, persist]
            b.set_tuning(knobs)
            assert b.tuning == knobs
            if mode == "run":
                b.run(steps)
            else:
                for _ in range(steps):
                    b.step()
            torch.cuda.synchronize()
            for s in sv:
                assert int(s.plan.scalars()[_lib.S_STATUS]) == 0
            assert int(sv[2].plan.scalars()[_lib.S_STEP]) == min(steps, 3)
            finals[persist, mode] = [s.q.clone() for s in sv]
            b.close()
    ref = finals[0, "run"]
    for key, got in finals.items():
        for a, c in zip(ref, got):
            assert torch.equal(a, c), key


@pytest.mark.gpu
def test_persistent_stage_not_available_reads_back_zero():
    """The persistent form needs FP32-bulk members of sensor width 4, lines
    of at most 512 nodes and all lines in one nodes-per-thread class of the
    sweeps; elsewhere the knob reads 0."""
    from hit_solver_b200.problems.riemann import RiemannConfig3, RiemannSolver

    cases = [
        [serving.make_solver(serving.Request(0, "riemann3", 40), "fp64")],
        [serving.make_solver(serving.Request(0, "riemann3", 640), "fp32-bulk")],
        [RiemannSolver(RiemannConfig3(nx=200, ny=64, precision="fp32-bulk"))],
        [RiemannSolver(RiemannConfig3(nx=64, ny=64, sensor_width=3, precision="fp32-bulk"))],
        [serving.make_solver(serving.Request(0, "riemann3", 64), "fp32-bulk"),
         serving.make_solver(serving.Request(1, "riemann3", 200), "fp32-bulk")],
    ]
    for sv in cases:
        b = Batch.from_plans([s.plan for s in sv], [s.q for s in sv])
        b.set_tuning([0, 0, 0, 0, 0, 1])
        assert b.tuning[_lib.TUNE_PERSISTENT] == 0
        b.close()
    s = serving.make_solver(serving.Request(0, "riemann3", 40), "fp32-bulk")
    s.plan.set_tuning([0, 0, 0, 0, 0, 1])
    assert s.plan.tuning[_lib.TUNE_PERSISTENT] == 0
