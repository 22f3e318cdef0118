"""Autotuner of the kernel variants.

Three kernel families have two compiled variants each: the x sweep, the y
sweep and the prepass; a fourth knob fuses each prepass into the following
sensor launch (single solves whose tiles all fit on the GPU at once), a
fifth picks the y sweep's tile shape (panels of 2 or 4 columns per CTA), and
a sixth runs each stage of a batch as one persistent launch (its members'
prepass, sensor and sweep work from one queue) instead of one launch per
phase.
The latency variant keeps more registers per thread
and suits launches that cannot fill the GPU (one 512^2 solve); the
throughput variant fits more CTAs per SM and suits launches over many solves.
Plans and batches start from a default picked by launch size.  The tuner
measures instead: it builds a copy of the batch (same descriptors, copies of
the member states, the members' time and step size), times a few steps of
each variant with per-launch CUDA events, keeps the faster variant of every
family, and applies it to the real batch.  The choice only changes speed, not
results, and is cached per batch signature (precision and each member's grid
and physics switches), so a serving loop that meets the same mix again pays
nothing.  The cache is also kept on disk (``HITB200_TUNE_CACHE``, default
``~/.cache/hit_solver_b200/tuning.json``; ``off`` disables it), keyed by the
signature, the GPU's name and the library build, so a later process on the
same GPU and build starts from the measured choice.
"""

from __future__ import annotations

import json
import os
import threading
from pathlib import Path

import torch

from . import _lib, core

_cache: dict = {}
_lock = threading.Lock()

# profile labels of each variant knob's kernels (hitb200_step_profile names)
_FAMILIES = {
    _lib.TUNE_SWEEP_X: ("sweep_x",),
    _lib.TUNE_SWEEP_Y: ("sweep_y",),
    _lib.TUNE_PREPASS: ("prepass", "hv_prepass"),
}
_VARIANT_KNOBS = (_lib.TUNE_SWEEP_X, _lib.TUNE_SWEEP_Y, _lib.TUNE_PREPASS)


def signature(descs) -> tuple:
    """Cache key: what the launch shapes and the work per cell depend on."""
    members = sorted(
        (d.nx, d.ny, d.periodic, d.scheme, d.sensor_width, int(d.viscosity > 0.0),
         int(d.forcing_on), int(d.drag_coefficient > 0.0), d.hv_interval)
        for d in descs)
    return (descs[0].precision, tuple(members))


def cache_path() -> Path | None:
    """The on-disk cache file, or None when disabled."""
    v = os.environ.get("HITB200_TUNE_CACHE", "")
    if v.lower() == "off":
        return None
    return Path(v) if v else Path.home() / ".cache" / "hit_solver_b200" / "tuning.json"


def _disk_key(key) -> str:
    """Signature plus what a measured choice depends on besides it: the GPU
    model and the library build (size and modification time of the .so)."""
    try:
        st = os.stat(_lib.LIB_PATH)
        build = f"{st.st_size}-{int(st.st_mtime)}"
    except OSError:
        build = "unknown"
    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return json.dumps([dev, build, key], separators=(",", ":"))


def _disk_load(dkey: str):
    path = cache_path()
    if path is None:
        return None
    try:
        data = json.loads(path.read_text())
    except (OSError, ValueError):
        return None
    v = data.get(dkey) if isinstance(data, dict) else None
    if isinstance(v, list) and len(v) == _lib.TUNE_COUNT and all(x in (0, 1) for x in v):
        return [int(x) for x in v]
    return None


def _disk_store(dkey: str, best) -> None:
    """Merge one entry into the cache file (written whole to a temporary file
    and renamed into place, so readers never see a partial file)."""
    path = cache_path()
    if path is None:
        return
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        try:
            data = json.loads(path.read_text())
            if not isinstance(data, dict):
                data = {}
        except (OSError, ValueError):
            data = {}
        data[dkey] = [int(x) for x in best]
        tmp = path.with_name(f"{path.name}.{os.getpid()}.tmp")
        tmp.write_text(json.dumps(data, indent=0, sort_keys=True))
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home: the in-memory cache still holds the choice


def _lookup(key, use_cache: bool):
    if not use_cache:
        return None
    with _lock:
        best = _cache.get(key)
    if best is None:
        best = _disk_load(_disk_key(key))
        if best is not None:
            with _lock:
                _cache[key] = best
    return best


def _remember(key, best, use_cache: bool) -> None:
    with _lock:
        _cache[key] = best
    if use_cache:
        _disk_store(_disk_key(key), best)


def _profile_ms(profile_fn, trials: int):
    """Mean device time per step of each knob's kernels, and of the whole
    step, over `trials` steps."""
    fam = {k: 0.0 for k in _FAMILIES}
    total = 0.0
    for _ in range(trials):
        for name, ms, _ in profile_fn():
            total += ms
            for k, names in _FAMILIES.items():
                if name in names:
                    fam[k] += ms
    return {k: v / trials for k, v in fam.items()}, total / trials


def _graph_ms(run_fn, steps: int) -> float:
    """Device time per step of `steps` graph-replayed steps."""
    st = torch.cuda.current_stream()
    run_fn(1)  # capture
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    run_fn(steps)
    b.record(st)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def _choose(profile_fn, set_fn, trials: int, run_fn=None) -> list[int]:
    """Variant knobs: each family's faster variant by per-launch times (fused
    sensor off, default y panels); then the y sweep's tile shape (the other
    panel width) by the y sweep's time; then, where run_fn can replay the
    plan's steps and the plan can fuse its prepasses into the sensors,
    whichever of fused / unfused gives the shorter graph-replayed step
    (launch gaps matter there)."""
    ms = {}
    for variant in (0, 1):
        set_fn([variant] * len(_VARIANT_KNOBS) + [0] * (_lib.TUNE_COUNT - len(_VARIANT_KNOBS)))
        profile_fn()  # warm-up step of this variant
        ms[variant] = _profile_ms(profile_fn, trials)[0]
    best = [0 if ms[0][k] <= ms[1][k] else 1 for k in _VARIANT_KNOBS]
    best += [0] * (_lib.TUNE_COUNT - len(best))
    ym = {}
    for panel in (0, 1):
        best[_lib.TUNE_Y_PANEL] = panel
        set_fn(best)
        profile_fn()
        ym[panel] = _profile_ms(profile_fn, trials)[0][_lib.TUNE_SWEEP_Y]
    best[_lib.TUNE_Y_PANEL] = 0 if ym[0] <= ym[1] else 1
    if run_fn is not None:
        step = {}
        for fused in (0, 1):
            best[_lib.TUNE_FUSED_SENSOR] = fused
            set_fn(best)
            step[fused] = _graph_ms(run_fn, max(4, 2 * trials))
        best[_lib.TUNE_FUSED_SENSOR] = 0 if step[0] <= step[1] else 1
    set_fn(best)
    return best


def _choose_persistent(batch, best: list[int], trials: int) -> list[int]:
    """Persistent stage launches or one launch per phase, whichever gives the
    shorter graph-replayed step (batches that cannot persist read the knob
    back as 0 and keep it off)."""
    trial = list(best)
    trial[_lib.TUNE_PERSISTENT] = 1
    batch.set_tuning(trial)
    if batch.tuning[_lib.TUNE_PERSISTENT] != 1:
        return best
    step = {}
    for persist in (0, 1):
        trial[_lib.TUNE_PERSISTENT] = persist
        batch.set_tuning(trial)
        step[persist] = _graph_ms(batch.run, max(4, 2 * trials))
    best = list(best)
    best[_lib.TUNE_PERSISTENT] = 0 if step[0] <= step[1] else 1
    batch.set_tuning(best)
    return best


def tune_batch(batch, trials: int = 3, use_cache: bool = True) -> list[int]:
    """Tune `batch` (a hit_solver_b200.batch.Batch with bound states)."""
    from .batch import Batch

    key = signature(batch.descs)
    best = _lookup(key, use_cache)
    if best is None:
        plans = [core.Plan(d) for d in batch.descs]
        states = [s.clone() for s in batch.states]
        scratch = Batch.from_plans(plans, states)
        try:
            for m, src in zip(scratch.members, batch.members):
                sc = src.scalars()
                m.set_time(sc[_lib.S_TIME], int(sc[_lib.S_STEP]), sc[_lib.S_DT], -1)
            best = _choose(scratch.step_profile, scratch.set_tuning, trials)
            best = _choose_persistent(scratch, best, trials)
        finally:
            scratch.close()
            del scratch, plans, states
            torch.cuda.synchronize()
        _remember(key, best, use_cache)
    batch.set_tuning(best)
    return best


def tune_plan(plan, q, trials: int = 3, use_cache: bool = True) -> list[int]:
    """Tune a single plan on a copy of its state q.  Plans whose forcing noise
    is uploaded per step (noise_mode 0) keep their default variants."""
    if plan.desc.forcing_on and plan.desc.noise_mode == 0:
        return plan.tuning
    key = signature([plan.desc]) + ("single",)
    best = _lookup(key, use_cache)
    if best is None:
        scratch = core.Plan(plan.desc)
        qc = q.clone()
        sc = plan.scalars()
        scratch.set_time(sc[_lib.S_TIME], int(sc[_lib.S_STEP]), sc[_lib.S_DT], -1)
        run = None
        if not (plan.desc.forcing_on and plan.desc.noise_mode == 0):
            run = lambda n: scratch.run(qc, n)  # noqa: E731
        best = _choose(lambda: scratch.step_profile(qc), scratch.set_tuning, trials, run)
        del scratch, qc
        torch.cuda.synchronize()
        _remember(key, best, use_cache)
    plan.set_tuning(best)
    return best


def clear_cache() -> None:
    with _lock:
        _cache.clear()
