"""Plans and device-array plumbing for the B200 backend.

A :class:`Plan` owns one ``hitb200_plan`` (one grid + physics descriptor and
its device scratch).  Arrays are torch CUDA tensors (float64 state
``[4, ny, nx]``, uint8/bool masks ``[ny, nx]``); they are passed to the C ABI
as raw device pointers on torch's current stream.
"""

from __future__ import annotations

import ctypes
import threading
import weakref

import torch

from . import _lib

_plan_cache: dict = {}
_cache_lock = threading.Lock()


def require_cuda() -> None:
    if not torch.cuda.is_available():
        raise RuntimeError("The b200 backend requires a CUDA device (B200, sm_100a)")
    _lib.load()


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def as_state(q, name: str = "state") -> torch.Tensor:
    """Return q as a contiguous float64 CUDA tensor of shape [4, ny, nx]."""
    if not isinstance(q, torch.Tensor):
        raise TypeError(f"{name} must be a torch CUDA tensor (the b200 backend's array type)")
    if q.device.type != "cuda":
        raise TypeError(f"{name} must live on a CUDA device")
    if q.dim() != 3 or q.shape[0] != 4:
        raise ValueError(f"{name} must have shape [4, ny, nx], got {tuple(q.shape)}")
    if q.dtype != torch.float64:
        q = q.to(torch.float64)
    return q.contiguous()


def as_field(a, shape, name: str, dtype=torch.float64) -> torch.Tensor:
    if not isinstance(a, torch.Tensor) or a.device.type != "cuda":
        raise TypeError(f"{name} must be a torch CUDA tensor")
    if tuple(a.shape) != tuple(shape):
        raise ValueError(f"{name} shape {tuple(a.shape)} does not match grid {tuple(shape)}")
    return a.to(dtype).contiguous()


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


class Plan:
    """One native plan.  Use :func:`plan_for` to share plans between the
    operator objects of one solve."""

    def __init__(self, desc: _lib.Desc):
        require_cuda()
        self.lib = _lib.load()
        self.desc = desc
        h = ctypes.c_void_p()
        torch.cuda.synchronize()
        _lib.check(self.lib.hitb200_plan_create(ctypes.byref(desc), ctypes.byref(h)))
        self.handle = h
        self._finalizer = weakref.finalize(self, Plan._destroy, self.lib, h.value)
        self.nx, self.ny = desc.nx, desc.ny

    @staticmethod
    def _destroy(lib, handle):
        if handle:
            lib.hitb200_plan_destroy(ctypes.c_void_p(handle))

    @property
    def shape(self):
        return (self.ny, self.nx)

    def device_bytes(self) -> int:
        return int(self.lib.hitb200_plan_device_bytes(ctypes.byref(self.desc)))

    # ---- operators --------------------------------------------------------
    def enforce(self, q: torch.Tensor) -> torch.Tensor:
        out = torch.empty_like(q)
        _lib.check(self.lib.hitb200_enforce(self.handle, q.data_ptr(), out.data_ptr(), stream_handle()))
        return out

    def sensor(self, q: torch.Tensor, enforce_first: bool) -> torch.Tensor:
        mask = torch.empty(self.shape, dtype=torch.uint8, device=q.device)
        _lib.check(self.lib.hitb200_sensor(self.handle, q.data_ptr(), mask.data_ptr(),
                                           int(enforce_first), stream_handle()))
        return mask.bool()

    def axis_derivative(self, q, mask, axis: int) -> torch.Tensor:
        out = torch.empty_like(q)
        m = mask.to(torch.uint8).contiguous()
        _lib.check(self.lib.hitb200_axis_derivative(self.handle, q.data_ptr(), m.data_ptr(), axis,
                                                    out.data_ptr(), stream_handle()))
        return out

    def rhs(self, q, terms=_lib.TERM_INVISCID, fx=None, fy=None) -> torch.Tensor:
        out = torch.empty_like(q)
        _lib.check(self.lib.hitb200_rhs(self.handle, q.data_ptr(), terms, ptr(fx), ptr(fy),
                                        out.data_ptr(), stream_handle()))
        return out

    def viscous_rhs(self, q) -> torch.Tensor:
        out = torch.empty_like(q)
        _lib.check(self.lib.hitb200_viscous_rhs(self.handle, q.data_ptr(), out.data_ptr(),
                                                stream_handle()))
        return out

    def hyperviscosity(self, q, active) -> torch.Tensor:
        out = torch.empty_like(q)
        a = active.to(torch.uint8).contiguous()
        _lib.check(self.lib.hitb200_hyperviscosity(self.handle, q.data_ptr(), a.data_ptr(),
                                                   out.data_ptr(), stream_handle()))
        return out

    def outflow_guard(self, q) -> torch.Tensor:
        out = q.clone()
        _lib.check(self.lib.hitb200_outflow_guard(self.handle, out.data_ptr(), stream_handle()))
        return out

    def stable_time_step(self, q, cfl, remaining=None) -> float:
        dt = ctypes.c_double()
        torch.cuda.current_stream().synchronize()
        _lib.check(self.lib.hitb200_stable_time_step(self.handle, q.data_ptr(), float(cfl),
                                                     _lib.none_to_nan(remaining), ctypes.byref(dt)))
        return dt.value

    def validate(self, q) -> int:
        torch.cuda.current_stream().synchronize()
        return int(self.lib.hitb200_validate(self.handle, q.data_ptr()))

    def forcing_update(self, q, noise, dt, target_power):
        fx = torch.empty(self.shape, dtype=torch.float64, device=q.device)
        fy = torch.empty_like(fx)
        _lib.check(self.lib.hitb200_forcing_update(self.handle, q.data_ptr(), ptr(noise), float(dt),
                                                   _lib.none_to_nan(target_power), fx.data_ptr(),
                                                   fy.data_ptr(), stream_handle()))
        return fx, fy

    # ---- time stepping ------------------------------------------------------
    def step(self, q, noise=None) -> None:
        _lib.check(self.lib.hitb200_step(self.handle, q.data_ptr(), ptr(noise), stream_handle()))

    def run(self, q, nsteps: int) -> None:
        _lib.check(self.lib.hitb200_run(self.handle, q.data_ptr(), int(nsteps), stream_handle()))

    def step_profile(self, q, noise=None):
        """One uncaptured step with per-launch CUDA events: list of
        (kernel, ms, algorithmic bytes)."""
        return profile_call(lambda ms, b, cap, cnt, names, size: self.lib.hitb200_step_profile(
            self.handle, q.data_ptr(), ptr(noise), ms, b, cap, cnt, names, size, stream_handle()))

    def set_time(self, time=0.0, step=0, dt=0.0, max_steps=-1) -> None:
        torch.cuda.current_stream().synchronize()
        _lib.check(self.lib.hitb200_set_time(self.handle, float(time), int(step), float(dt),
                                             int(max_steps)))

    def scalars(self, n: int = _lib.S_COUNT) -> list[float]:
        buf = (ctypes.c_double * n)()
        _lib.check(self.lib.hitb200_read_scalars(self.handle, buf, n))
        return list(buf)

    def set_noise_stream(self, pcg64_state: dict) -> None:
        """Continue a NumPy PCG64 stream (``bit_generator.state``) on the device
        (noise_mode 2 plans)."""
        st = pcg64_state["state"]
        mask = (1 << 64) - 1
        words = (ctypes.c_uint64 * 4)(st["state"] & mask, st["state"] >> 64, st["inc"] & mask,
                                      st["inc"] >> 64)
        _lib.check(self.lib.hitb200_set_noise_stream(self.handle, words))

    def noise_stream(self) -> dict:
        """The device noise stream's position as a NumPy PCG64 state dict."""
        words = (ctypes.c_uint64 * 4)()
        _lib.check(self.lib.hitb200_get_noise_stream(self.handle, words))
        return {"bit_generator": "PCG64",
                "state": {"state": words[0] | (words[1] << 64), "inc": words[2] | (words[3] << 64)},
                "has_uint32": 0, "uinteger": 0}

    def save_state_block(self):
        """The whole device scalar block (time, step, controller and forcing
        state, OU potential): with the state q, a checkpoint of the solve."""
        import numpy as np

        n = int(self.lib.hitb200_state_block_size())
        buf = (ctypes.c_double * n)()
        _lib.check(self.lib.hitb200_save_state_block(self.handle, buf, n))
        return np.array(buf, dtype=np.float64)

    def load_state_block(self, block) -> None:
        import numpy as np

        block = np.ascontiguousarray(block, dtype=np.float64)
        n = int(self.lib.hitb200_state_block_size())
        if block.shape != (n,):
            raise ValueError(f"state block must hold {n} doubles")
        _lib.check(self.lib.hitb200_load_state_block(
            self.handle, block.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))

    @property
    def tuning(self) -> list[int]:
        """Kernel variant knobs (see hit_solver_b200.autotune)."""
        return get_tuning(self.lib.hitb200_plan_get_tuning, self.handle)

    def set_tuning(self, knobs) -> None:
        set_tuning(self.lib.hitb200_plan_set_tuning, self.handle, knobs)

    def diagnostics(self, q) -> list[float]:
        buf = (ctypes.c_double * 17)()
        torch.cuda.current_stream().synchronize()
        _lib.check(self.lib.hitb200_diagnostics(self.handle, q.data_ptr(), buf, 17))
        return list(buf)


def get_tuning(fn, handle) -> list[int]:
    buf = (ctypes.c_int32 * _lib.TUNE_COUNT)()
    _lib.check(fn(handle, buf, _lib.TUNE_COUNT))
    return list(buf)


def set_tuning(fn, handle, knobs) -> None:
    knobs = list(knobs)
    buf = (ctypes.c_int32 * len(knobs))(*[int(k) for k in knobs])
    _lib.check(fn(handle, buf, len(knobs)))


def profile_call(fn, cap: int = 64):
    ms = (ctypes.c_float * cap)()
    by = (ctypes.c_double * cap)()
    cnt = ctypes.c_int32()
    names = ctypes.create_string_buffer(4096)
    _lib.check(fn(ms, by, cap, ctypes.byref(cnt), names, 4096))
    labels = names.value.decode().split("\n")
    return [(labels[i], float(ms[i]), float(by[i])) for i in range(min(cnt.value, cap))]


def plan_for(desc: _lib.Desc) -> Plan:
    """Shared plan per descriptor (operator objects of one solve share one)."""
    key = desc.key()
    with _cache_lock:
        p = _plan_cache.get(key)
        if p is None:
            p = Plan(desc)
            _plan_cache[key] = p
        return p


def clear_plan_cache() -> None:
    with _cache_lock:
        _plan_cache.clear()
