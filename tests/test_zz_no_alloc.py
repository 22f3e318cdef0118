"""hitb200_stable_time_step_noalloc: the plan-less, allocation-free time step.

Some callers cannot allocate device memory where they need the time step (a
plan's creation calls cudaMalloc; its destruction calls cudaFree, which
synchronises the device).  This entry point reduces into a static device array
shared by every call on a device, so this file is collected last: it checks
that two calls in a row, after whatever the other test files ran, agree with
the plan-based hitb200_stable_time_step on the same states.
"""

import ctypes
import math

import numpy as np
import pytest
import torch

from hit_solver_b200 import _lib, core
from hit_solver_b200.descs import grid_desc
from hit_solver_b200.domain import Domain2D
from oracle import hit_oracle as O
from tests.gpu_util import periodic_state

G = 1.4
RTOL = 1e-14  # same per-cell formula and an exact maximum


def _noalloc(q, dom, cfl, remaining, out):
    lib = _lib.load()
    _lib.check(lib.hitb200_stable_time_step_noalloc(
        q.data_ptr(), dom.nx, dom.ny, dom.dx, dom.dy, G, cfl,
        _lib.none_to_nan(remaining), out.data_ptr(), core.stream_handle()))
    return float(out.item())


def _plan(dom, periodic):
    return core.Plan(grid_desc(dom, G, periodic, "fp64"))


def _close(a, b):
    return abs(a - b) <= RTOL * abs(b)


def test_noalloc_rejects_before_any_device_work():
    lib = _lib.load()
    out = ctypes.c_double()
    addr = ctypes.addressof(out)
    # 1056 x 1024 cells = 33 x 32 tiles, more than the scratch's 1024
    st = lib.hitb200_stable_time_step_noalloc(addr, 1056, 1024, 1e-3, 1e-3, G, 0.4, math.nan, addr, None)
    assert st == _lib.ERR_UNSUPPORTED
    assert "1024" in lib.hitb200_status_string(st).decode()
    nan = math.nan
    assert lib.hitb200_stable_time_step_noalloc(None, 8, 8, 1.0, 1.0, G, 0.4, nan, addr, None) == _lib.ERR_INVALID
    assert lib.hitb200_stable_time_step_noalloc(addr, 0, 8, 1.0, 1.0, G, 0.4, nan, addr, None) == _lib.ERR_INVALID
    assert lib.hitb200_stable_time_step_noalloc(addr, 8, 8, 1.0, 1.0, G, -1.0, nan, addr, None) == _lib.ERR_INVALID
    # tile counts formed in 64 bits: near INT32_MAX cells per line is rejected, not overflowed
    big = 2**31 - 1
    assert lib.hitb200_stable_time_step_noalloc(addr, big, big, 1.0, 1.0, G, 0.4, nan, addr, None) == _lib.ERR_UNSUPPORTED
    assert lib.hitb200_stable_time_step_noalloc(addr, big, 1, 1.0, 1.0, G, 0.4, nan, addr, None) == _lib.ERR_UNSUPPORTED


@pytest.mark.gpu
def test_noalloc_matches_plan_time_step():
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    riemann = Domain2D(0.0, 1.0, 0.0, 1.0, 64, 64)
    hit = Domain2D(0.0, 2 * np.pi, 0.0, 2 * np.pi, 96, 80)
    cases = [(riemann, False, O.enforce(O.riemann_initial_state(3, 64, 64, 0.8, 0.8, G), G)),
             (hit, True, periodic_state(96, 80))]
    for dom, periodic, qh in cases:
        q = torch.from_numpy(np.ascontiguousarray(qh)).cuda()
        plan = _plan(dom, periodic)
        for cfl, rem in ((0.4, None), (0.3, 1e-6)):
            ref = plan.stable_time_step(q, cfl, rem)
            first = _noalloc(q, dom, cfl, rem, out)
            second = _noalloc(q, dom, cfl, rem, out)
            assert _close(first, ref), (first, ref)
            assert _close(second, ref), (second, ref)


@pytest.mark.gpu
def test_noalloc_largest_grid_twice():
    # 1024 x 1024 cells: exactly the 1024 tiles the static scratch holds
    n = 1024
    dom = Domain2D(0.0, 1.0, 0.0, 1.0, n, n)
    gen = torch.Generator(device="cuda").manual_seed(7)
    rho = 1.0 + 0.5 * torch.rand((n, n), generator=gen, device="cuda", dtype=torch.float64)
    u = torch.randn((n, n), generator=gen, device="cuda", dtype=torch.float64)
    v = torch.randn((n, n), generator=gen, device="cuda", dtype=torch.float64)
    p = 0.5 + torch.rand((n, n), generator=gen, device="cuda", dtype=torch.float64)
    q = torch.stack([rho, rho * u, rho * v, p / (G - 1.0) + 0.5 * rho * (u * u + v * v)]).contiguous()
    ref = _plan(dom, False).stable_time_step(q, 0.4, None)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    assert _close(_noalloc(q, dom, 0.4, None, out), ref)
    assert _close(_noalloc(q, dom, 0.4, None, out), ref)


def _random_state(nx, ny, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    shape = (ny, nx)
    rho = 1.0 + 0.5 * torch.rand(shape, generator=gen, device="cuda", dtype=torch.float64)
    u = torch.randn(shape, generator=gen, device="cuda", dtype=torch.float64)
    v = torch.randn(shape, generator=gen, device="cuda", dtype=torch.float64)
    p = 0.5 + torch.rand(shape, generator=gen, device="cuda", dtype=torch.float64)
    return torch.stack([rho, rho * u, rho * v, p / (G - 1.0) + 0.5 * rho * (u * u + v * v)]).contiguous()


@pytest.mark.gpu
def test_noalloc_queued_calls_without_sync():
    # Calls queued back to back on one stream, each with its own state and
    # output slot and no host synchronisation between them: the ticket counter
    # each call leaves at zero serves the next one.  The 33 x 1000 grid has a
    # ragged last tile in both directions (2 x 32 tiles).
    lib = _lib.load()
    dom = Domain2D(0.0, 1.0, 0.0, 2.0, 33, 1000)
    states = [_random_state(33, 1000, seed) for seed in (1, 2, 3)]
    out = torch.full((len(states),), -1.0, dtype=torch.float64, device="cuda")
    for k, q in enumerate(states):
        _lib.check(lib.hitb200_stable_time_step_noalloc(
            q.data_ptr(), dom.nx, dom.ny, dom.dx, dom.dy, G, 0.4, math.nan,
            out.data_ptr() + 8 * k, core.stream_handle()))
    torch.cuda.synchronize()
    plan = _plan(dom, False)
    for k, q in enumerate(states):
        ref = plan.stable_time_step(q, 0.4, None)
        assert _close(float(out[k]), ref), (k, float(out[k]), ref)


@pytest.mark.gpu
def test_noalloc_nan_cell_gives_nan():
    # np.max propagates NaN, so the reference's time step of a state with a
    # NaN cell is NaN; the maximum here carries it the same way.
    dom = Domain2D(0.0, 1.0, 0.0, 1.0, 96, 80)
    q = _random_state(96, 80, 5)
    q[1, 41, 17] = float("nan")
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    assert math.isnan(_noalloc(q, dom, 0.4, None, out))
    q[1, 41, 17] = 0.0
    assert math.isfinite(_noalloc(q, dom, 0.4, None, out))
