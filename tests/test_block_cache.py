"""Device block cache of the library (plan arenas and batch tables).

A destroyed plan or batch keeps its device block for later plans and batches
of the same device (hitb200_release_cached_blocks frees them).  A plan whose
arena is a reused block must compute exactly what a plan on a fresh block
computes: every buffer a step reads is written first, whatever the block
held before.
"""

import gc

import pytest
import torch

from hit_solver_b200 import _lib, serving
from hit_solver_b200.batch import Batch

GRANULE = 2 << 20


def test_release_with_nothing_cached():
    lib = _lib.load()
    assert lib.hitb200_release_cached_blocks() == _lib.OK
    assert lib.hitb200_cached_block_bytes() == 0


def _run(req, steps):
    s = serving.make_solver(req, "fp32-bulk")
    s.advance(steps)
    torch.cuda.synchronize()
    return s, s.q.clone()


@pytest.mark.gpu
@pytest.mark.parametrize("req", [
    serving.Request(0, "riemann3", 96, split=0.45),
    serving.Request(1, "hit", 64, seed=3, mach=0.3, steps=10 ** 6),
], ids=["riemann3_96", "hit_64"])
def test_reused_arena_gives_identical_run(req):
    lib = _lib.load()
    lib.hitb200_release_cached_blocks()
    s, first = _run(req, 6)
    want = s.plan.device_bytes()
    assert lib.hitb200_cached_block_bytes() == 0
    del s
    gc.collect()
    held = lib.hitb200_cached_block_bytes()
    assert want <= held < want + GRANULE
    # fill the cached block with garbage through a plan of another problem
    # first, so that the second run cannot see the first run's leftovers only
    other = serving.make_solver(serving.Request(2, "riemann6", 96, split=0.6), "fp32-bulk")
    other.advance(3)
    torch.cuda.synchronize()
    del other
    gc.collect()
    s2, second = _run(req, 6)
    assert lib.hitb200_cached_block_bytes() < held + GRANULE
    assert torch.equal(first, second)
    assert int(s2.plan.scalars()[_lib.S_STATUS]) == 0
    del s2
    gc.collect()
    lib.hitb200_release_cached_blocks()
    assert lib.hitb200_cached_block_bytes() == 0


@pytest.mark.gpu
def test_batch_tables_return_to_the_cache():
    lib = _lib.load()
    lib.hitb200_release_cached_blocks()
    sv = [serving.make_solver(serving.Request(i, "riemann3", 64 + 32 * i, split=0.5), "fp32-bulk")
          for i in range(3)]
    outs = []
    for _ in range(2):
        for s in sv:
            s.plan.set_time(0.0, 0, s.plan.scalars()[_lib.S_DT])
        qs = [s.q.clone() for s in sv]
        b = Batch.from_plans([s.plan for s in sv], qs)
        b.run(4)
        torch.cuda.synchronize()
        b.close()
        outs.append(qs)
        assert lib.hitb200_cached_block_bytes() >= GRANULE  # the tables' block
    for a, c in zip(*outs):
        assert torch.equal(a, c)
    lib.hitb200_release_cached_blocks()
    assert lib.hitb200_cached_block_bytes() == 0
