"""Batched form: many independent solves (mixed grid sizes, HIT and Riemann)
advanced together, one launch per kernel of the step for all of them.

Each member keeps its own resident state tensor and device scalar block (time,
dt, forcing state, ...); the kernels take a per-solve descriptor table and a
work list whose CTAs cover every member's tiles and lines, so small and large
grids share the GPU in the same launch.  Steps are replayed from one captured
CUDA graph; a member whose time reached tfinal (or max_steps) turns into a
device-side no-op while the others continue.
"""

from __future__ import annotations

import ctypes
import weakref

import torch

from . import _lib, core


class MemberPlan:
    """View of one batch member's plan (time / scalar access)."""

    def __init__(self, lib, handle):
        self.lib = lib
        self.handle = ctypes.c_void_p(handle)

    def set_time(self, time=0.0, step=0, dt=0.0, max_steps=-1) -> None:
        torch.cuda.current_stream().synchronize()
        _lib.check(self.lib.hitb200_set_time(self.handle, float(time), int(step), float(dt),
                                             int(max_steps)))

    def scalars(self, n: int = _lib.S_COUNT) -> list[float]:
        buf = (ctypes.c_double * n)()
        _lib.check(self.lib.hitb200_read_scalars(self.handle, buf, n))
        return list(buf)

    def copy_scalars_async(self, dst: torch.Tensor, n: int = _lib.S_COUNT) -> None:
        _lib.check(self.lib.hitb200_copy_scalars_async(self.handle, dst.data_ptr(), n,
                                                       core.stream_handle()))


class Batch:
    def __init__(self, descs):
        core.require_cuda()
        self.lib = _lib.load()
        n = len(descs)
        if n == 0:
            raise ValueError("batch needs at least one descriptor")
        arr = (_lib.Desc * n)(*descs)
        h = ctypes.c_void_p()
        torch.cuda.synchronize()
        _lib.check(self.lib.hitb200_batch_create(arr, n, ctypes.byref(h)))
        self.handle = h
        self._finalizer = weakref.finalize(self, Batch._destroy, self.lib, h.value)
        self.descs = list(descs)
        self.members = [MemberPlan(self.lib, self.lib.hitb200_batch_plan(h, i)) for i in range(n)]
        self.states: list[torch.Tensor] = []

    @classmethod
    def from_plans(cls, plans, states) -> "Batch":
        """A batch over existing plans (hitb200_batch_from_plans) with their
        resident states bound.  The plans stay owned by their Plan objects:
        close() hands them back for use alone or in a later batch."""
        self = cls.__new__(cls)
        self.lib = _lib.load()
        n = len(plans)
        if n == 0:
            raise ValueError("batch needs at least one plan")
        arr = (ctypes.c_void_p * n)(*[p.handle.value for p in plans])
        h = ctypes.c_void_p()
        torch.cuda.synchronize()
        _lib.check(self.lib.hitb200_batch_from_plans(arr, n, ctypes.byref(h)))
        self.handle = h
        self._plans = list(plans)  # the plans outlive the batch
        self._finalizer = weakref.finalize(self, Batch._destroy, self.lib, h.value)
        self.descs = [p.desc for p in plans]
        self.members = [MemberPlan(self.lib, p.handle.value) for p in plans]
        self.states = []
        self.bind(states)
        return self

    def close(self) -> None:
        """Destroy the native batch now (waits for the device)."""
        self._finalizer()

    @staticmethod
    def _destroy(lib, handle):
        if handle:
            lib.hitb200_batch_destroy(ctypes.c_void_p(handle))

    def __len__(self) -> int:
        return len(self.members)

    @property
    def cells(self) -> int:
        return sum(d.nx * d.ny for d in self.descs)

    def bind(self, states) -> None:
        if len(states) != len(self.members):
            raise ValueError("one state per member is required")
        for s, d in zip(states, self.descs):
            if tuple(s.shape) != (4, d.ny, d.nx) or s.dtype != torch.float64 or not s.is_cuda:
                raise ValueError("member state must be a float64 CUDA tensor [4, ny, nx]")
            if not s.is_contiguous():
                raise ValueError("member state must be contiguous")
        self.states = list(states)
        ptrs = (ctypes.c_void_p * len(states))(*[s.data_ptr() for s in states])
        torch.cuda.synchronize()
        _lib.check(self.lib.hitb200_batch_bind(self.handle, ptrs))

    def step(self) -> None:
        _lib.check(self.lib.hitb200_batch_step(self.handle, core.stream_handle()))

    def run(self, nsteps: int) -> None:
        _lib.check(self.lib.hitb200_batch_run(self.handle, int(nsteps), core.stream_handle()))

    @property
    def tuning(self) -> list[int]:
        """Kernel variant knobs (see hit_solver_b200.autotune)."""
        return core.get_tuning(self.lib.hitb200_batch_get_tuning, self.handle)

    def set_tuning(self, knobs) -> None:
        core.set_tuning(self.lib.hitb200_batch_set_tuning, self.handle, knobs)

    def autotune(self, trials: int = 3) -> list[int]:
        """Pick each kernel family's variant by timing both on a copy of this
        batch (hit_solver_b200.autotune.tune_batch)."""
        from .autotune import tune_batch

        return tune_batch(self, trials=trials)

    def step_profile(self):
        return core.profile_call(lambda ms, b, cap, cnt, names, size:
                                 self.lib.hitb200_batch_step_profile(
                                     self.handle, ms, b, cap, cnt, names, size,
                                     core.stream_handle()))
