#!/usr/bin/env python
"""Throughput of the HIT_Solver RHS / SSP-RK3 hot path on B200.

Workload (the reference's headline Riemann case): Lax-Liu configuration 3 on
a 512 x 512 grid, hybrid compact/WENO7 scheme, sensor width 4, jump
threshold 0.025, no shear term, hyperviscosity mn = 0.001 every step,
CFL 0.4 (dt fixed from the initial state), outflow guard cells 2.
One step = one full SSP-RK3 step (three RHS evaluations, clean filters,
hyperviscosity).  Metric: cell-updates/s (cells x steps / s).

  value       FP32-bulk form (FP32 stencil/WENO/flux arithmetic, FP64 state),
              one solve, device-timed with CUDA events, L2 flushed before
              every timed step (the solve's working set would otherwise stay
              in the 126 MB L2).
  plain_fp64  the same solve in the plain FP64 form.
  batched     B independent 512^2 solves (quadrant-state sweep of the split
              point) advanced by one launch per kernel of the step.
  e2e         the public API with host buffers: the initial state uploaded
              from pinned memory, each step's scalar record (time, status)
              read back, the final state downloaded, all inside the timed
              region.
  roofline    the step's dominant kernel: algorithmic bytes per launch /
              its CUDA-event launch time; ``step``: the whole step's
              algorithmic 256 B per cell-update over the measured step time.
  cpu_baseline  the CPU oracle (NumPy FP64 restatement of the reference
              algorithm) on a bounded number of steps of the same workload.
  spectra     shell spectra of 64 resident 512^2 snapshots per step (the
              per-snapshot work of HIT2DSpectra.compute), snapshots/s, with
              its phases against the HBM peak and the oracle on 3 snapshots.

Launch:  python bench.py [--gpus N --steps K --warmup W]; for N > 1 under
torchrun each rank runs its own replica (the solve does not shard).
``--impl reference`` times the reference algorithm's CPU implementation
(the oracle port) on the host cores instead.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s per RK3 step (Riemann config 3, 512x512, hybrid WENO7/compact)"
NX = NY = 512
WORKLOAD = {"workload": "riemann_config3_512x512_hybrid_hv1_cfl0.4", "nx": NX, "ny": NY,
            "scheme": "hybrid", "sensor_width": 4, "jump_threshold": 0.025, "shear": None,
            "hyperviscosity_mn": 0.001, "hyperviscosity_interval": 1, "cfl": 0.4,
            "guard_cells": 2, "precision": "fp32-bulk (fp64 state)"}
FALLBACK_HBM_GBS = 6650.0
STEP_BYTES_PER_CELL = 256  # 8 FP64 state vectors (4 components) per SSP-RK3 step


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=("b200", "reference"), default="b200")
    p.add_argument("--batch", type=int, default=8, help="solves in the batched measurement")
    p.add_argument("--cpu-steps", type=int, default=3, help="oracle steps in the cpu_baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--ref-procs", type=int, default=0,
                   help="reference arm: host processes (0: one per core, at most 32)")
    p.add_argument("--ensemble", type=int, default=64, help="solves in the ensemble leg (0: skip)")
    p.add_argument("--spectra", type=int, default=64,
                   help="snapshots per step in the shell-spectra leg (0: skip)")
    p.add_argument("--serve-requests", type=int, default=24,
                   help="requests in the serving measurement (0: skip)")
    p.add_argument("--serve-rate", type=float, default=20.0, help="mean arrivals per second")
    p.add_argument("--serve-round", type=int, default=16, help="steps between admission points")
    p.add_argument("--only", choices=("all", "single"), default="all",
                   help="single: only the FP32-bulk single-solve steps, no JSON line "
                        "(a short launch sequence for profilers)")
    return p.parse_args()


# ----------------------------------------------------------------------------------
# distributed plumbing (replicas only: no data-path collective)
# ----------------------------------------------------------------------------------
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def dist_finish(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ----------------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region:
    NVML polled from a thread every 10 ms (falls back to nvidia-smi -lms 200)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown"}

    def __init__(self, cuda_index: int):
        self.cuda_index = cuda_index
        self.samples = []
        self.max_mhz = None
        self.proc = None
        self.thread = None
        self.path = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def __enter__(self):
        import threading

        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop = threading.Event()

            def poll():
                while not self.stop.is_set():
                    try:
                        mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((float(mhz), int(bits)))
                    except Exception:
                        pass
                    self.stop.wait(0.01)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.path = Path(tempfile.mkstemp(prefix="clocks_", suffix=".csv")[1])
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.cuda_index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.thread is not None:
            if not self.samples:
                return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"]}
            reasons = sorted({name for _, bits in self.samples
                              for bit, name in self.REASONS.items() if bits & bit})
            return {"sm_mhz": statistics.median(m for m, _ in self.samples),
                    "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(self.samples), "source": "nvml"}
        if self.proc is None or self.path is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi"}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel: str):
    """Per-launch DRAM traffic of the dominant kernel from the committed ncu
    summary (profiles/ncu_traffic.json), scaled to this workload, or None."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    try:
        data = json.loads(p.read_text())
        entry = data.get(kernel)
        if entry is None:
            return None
        return float(entry["bytes_per_cell"]) * NX * NY
    except (KeyError, ValueError, TypeError):
        return None


# ----------------------------------------------------------------------------------
# b200 arm
# ----------------------------------------------------------------------------------
def make_solver(precision: str, x_split: float = 0.5):
    from hit_solver_b200.problems.riemann import RiemannConfig3, RiemannSolver

    cfg = RiemannConfig3(nx=NX, ny=NY, x_split=x_split, y_split=x_split, shear_threshold=None,
                         precision=precision)
    solver = RiemannSolver(cfg)
    # timing runs continue past tfinal: no step limit on the device
    solver.plan.set_time(0.0, 0, solver.dt, -1)
    return solver


def flush_buffer():
    import torch

    return torch.empty(320 * 2 ** 20 // 4, dtype=torch.float32, device="cuda")  # 320 MB > L2


def timed_steps(advance, steps: int, flush) -> float:
    """Sum of per-step CUDA-event times with an L2 flush before each step."""
    import torch

    st = torch.cuda.current_stream()
    total = 0.0
    evs = []
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        advance()
        b.record(st)
        evs.append((a, b))
    torch.cuda.synchronize()
    for a, b in evs:
        total += a.elapsed_time(b)
    return total / 1e3


def profile_steps(profile_fn, nprof: int, flush):
    """Per-kernel-type mean launch time and algorithmic bytes over nprof
    uncaptured steps, each after an L2 flush."""
    per = {}
    for _ in range(nprof):
        flush.zero_()
        for name, ms, by in profile_fn():
            d = per.setdefault(name, {"ms": 0.0, "bytes": 0.0, "launches": 0})
            d["ms"] += ms
            d["bytes"] += by
            d["launches"] += 1
    for d in per.values():
        d["ms_per_launch"] = d["ms"] / d["launches"]
        d["bytes_per_launch"] = d["bytes"] / d["launches"]
        d["ms_per_step"] = d["ms"] / nprof
    return per


def run_b200(args, world, rank, local):
    import numpy as np
    import torch

    from hit_solver_b200 import _lib
    from hit_solver_b200.batch import Batch
    from hit_solver_b200.problems.riemann import riemann_descriptor, RiemannConfig3

    torch.cuda.set_device(local)
    K, W = args.steps, max(args.warmup, 3)
    flush = flush_buffer()
    cells = NX * NY

    from hit_solver_b200 import autotune

    tuning = {}
    # ---- FP32-bulk single solve (value) ----
    s32 = make_solver("fp32-bulk")
    tuning["single_fp32"] = autotune.tune_plan(s32.plan, s32.q)
    s32.advance(W)
    torch.cuda.synchronize()
    dist_barrier(world)
    with ClockSampler(local) as clk:
        t32 = timed_steps(lambda: s32.advance(1), K, flush)
        torch.cuda.synchronize()
    dist_barrier(world)
    t32 = dist_max(t32, world)
    if args.only == "single":
        return None
    launches_per_step = len(s32.plan.step_profile(s32.q))

    # ---- plain FP64 single solve ----
    s64 = make_solver("fp64")
    tuning["plain_fp64"] = autotune.tune_plan(s64.plan, s64.q)
    s64.advance(W)
    t64 = dist_max(timed_steps(lambda: s64.advance(1), K, flush), world)

    # ---- batched: B independent solves, split points swept over [0.3, 0.8] ----
    B = max(1, args.batch)
    descs, states, dts = [], [], []
    for i in range(B):
        split = 0.3 + 0.5 * i / max(B - 1, 1)
        cfg = RiemannConfig3(nx=NX, ny=NY, x_split=split, y_split=split, shear_threshold=None,
                             precision="fp32-bulk")
        sv = make_solver("fp32-bulk", split)
        descs.append(riemann_descriptor(cfg))
        states.append(sv.q.clone())
        dts.append(sv.dt)
        del sv
    batch = Batch(descs)
    batch.bind(states)
    for m, dt in zip(batch.members, dts):
        m.set_time(0.0, 0, dt, -1)
    tuning["batched"] = batch.autotune()
    batch.run(W)
    tb = dist_max(timed_steps(lambda: batch.run(1), max(K // 4, 5), flush), world)
    kb = max(K // 4, 5)
    batch.close()
    del batch, states

    # ---- 512^2 production HIT: plain FP64 single solve vs FP32-bulk batch ----
    hit = hit_forms(K, W, B, flush, world)
    dropin = dropin_hit_run() if rank == 0 else None
    hit["tuning"] = hit.pop("_tuning")
    ens = ensemble_run(K, W, flush, world, args.ensemble) if args.ensemble > 0 else None
    if ens is not None:
        ens["speedup_vs_plain_fp64_hit_512"] = ens["value"] / hit["plain_fp64"]["value"]

    # ---- shell spectra of resident snapshots (HIT2DSpectra's per-snapshot work) ----
    spectra = (spectra_run(K, W, flush, world, args.spectra,
                           rank == 0 and world == 1 and not args.no_cpu_baseline)
               if args.spectra > 0 else None)

    # ---- initial states: host vs device construction at 1024^2 ----
    init = initial_state_run() if rank == 0 else None

    # ---- serving: a seeded Poisson stream through the continuous-batching loop ----
    serve = serving_run(args) if args.serve_requests > 0 else None

    # ---- roofline of the dominant kernel (FP32-bulk solve) ----
    per = profile_steps(lambda: s32.plan.step_profile(s32.q), 5, flush)
    dom_name = max(per, key=lambda k: per[k]["ms_per_step"])
    dom = per[dom_name]
    peak, peak_kind = measured_peak()
    achieved = dom["bytes_per_launch"] / (dom["ms_per_launch"] / 1e3) / 1e9

    # ---- e2e through the public API with host buffers ----
    q_host = s32.q.detach().cpu().pin_memory()
    out_host = torch.empty_like(q_host).pin_memory()
    scal_host = torch.empty((K, _lib.S_COUNT), dtype=torch.float64).pin_memory()
    e2e_solver = make_solver("fp32-bulk")
    q_dev = e2e_solver.q
    e2e_solver.advance(W)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    q_dev.copy_(q_host, non_blocking=True)
    for k in range(K):
        e2e_solver.plan.run(q_dev, 1)
        e2e_solver.plan.lib.hitb200_copy_scalars_async(e2e_solver.plan.handle,
                                                       scal_host[k].data_ptr(), _lib.S_COUNT,
                                                       st.cuda_stream)
    out_host.copy_(q_dev, non_blocking=True)
    b.record(st)
    torch.cuda.synchronize()
    te2e = dist_max(a.elapsed_time(b) / 1e3, world)
    state_bytes = 4 * cells * 8
    if int(scal_host[:, _lib.S_STATUS].max()) & 1:
        raise FloatingPointError("non-finite state during the e2e run")

    # ---- CPU baseline (oracle port, rank 0 at N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_steps)

    if rank != 0:
        return None
    value = world * cells * K / t32
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": 1e3 * t32 / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 (fp64 state)",
        "data": "synthetic: the reference's own Riemann config-3 initial state (no dataset)",
        "config": {**WORKLOAD, "parallelism": f"replicas x{world}" if world > 1 else "single",
                   "l2": "flushed (320 MB write) before every timed step"},
        "plain_fp64": {"value": world * cells * K / t64, "ms_per_step": 1e3 * t64 / K,
                       "dtype": "fp64"},
        "batched": {"value": world * B * cells * kb / tb, "ms_per_step": 1e3 * tb / kb,
                    "solves": B, "dtype": "fp32 (fp64 state)",
                    "speedup_vs_plain_fp64": (B * cells * kb / tb) / (cells * K / t64)},
        "batched_hit": hit,
        "dropin_hit": dropin,
        # the headline's companions in one place: the batched FP32 form against
        # the plain FP64 single solve on 512^2 production HIT (the target
        # ratio, 5x), the plain FP64 Riemann solve, and the drop-in HIT path
        "batched_vs_plain": {
            "batched_fp32_hit_cell_updates_per_s": hit["batched_fp32"]["value"],
            "plain_fp64_hit_cell_updates_per_s": hit["plain_fp64"]["value"],
            "batched_vs_plain_fp64_hit": hit["speedup_batched_vs_plain"],
            "plain_fp64_riemann_cell_updates_per_s": world * cells * K / t64,
            "dropin_hit_ms_per_step": None if dropin is None else dropin["numpy"]["ms_per_step"],
        },
        "ensemble": ens,
        "serving": serve,
        "spectra": spectra,
        "initial_states": init,
        "e2e": {"value": world * cells * K / te2e, "unit": "cell-updates/s",
                "h2d_bytes_per_step": state_bytes / K,
                "d2h_bytes_per_step": 8 * _lib.S_COUNT + state_bytes / K},
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_kind == "measured" else "fallback 6.65 TB/s",
                     "traffic": ncu_traffic(dom_name),
                     "bytes_per_launch": dom["bytes_per_launch"],
                     "ms_per_launch": dom["ms_per_launch"],
                     "kernels": {k: {"ms_per_step": round(v["ms_per_step"], 5),
                                     "ms_per_launch": round(v["ms_per_launch"], 5),
                                     "gbs": round(v["bytes_per_launch"] / (v["ms_per_launch"] / 1e3) / 1e9, 1)
                                     if v["bytes_per_launch"] > 0 else None}
                                 for k, v in sorted(per.items(), key=lambda kv: -kv[1]["ms_per_step"])},
                     # the whole step against the same peak: 8 FP64 state
                     # vectors of SSP-RK3 per cell-update (256 B)
                     "kernels_mode": "each kernel timed alone: one uncaptured step with CUDA "
                                     "events between launches (no programmatic-launch overlap); "
                                     "their sum is kernels_sum_ms_per_step, the graph-replayed "
                                     "step is ms_per_step",
                     "kernels_sum_ms_per_step": round(sum(v["ms_per_step"] for v in per.values()), 5),
                     "step": {"bytes_per_cell_update": STEP_BYTES_PER_CELL,
                              "plain_fp64_hit_gbs": STEP_BYTES_PER_CELL * hit["plain_fp64"]["value"] / 1e9,
                              "batched_fp32_hit_gbs": STEP_BYTES_PER_CELL * hit["batched_fp32"]["value"] / 1e9,
                              "batched_vs_plain_fp64_hit": hit["speedup_batched_vs_plain"],
                              "single_gbs": STEP_BYTES_PER_CELL * cells * K / t32 / 1e9,
                              "single_frac": STEP_BYTES_PER_CELL * cells * K / t32 / 1e9 / peak,
                              "batched_gbs": STEP_BYTES_PER_CELL * B * cells * kb / tb / 1e9,
                              "batched_frac": STEP_BYTES_PER_CELL * B * cells * kb / tb / 1e9 / peak}},
        "tuning": {"knobs": "sweep_x, sweep_y, prepass: 0 latency / 1 throughput variant; "
                            "fused prepass + sensor; y panel: 0 default / 1 other width; "
                            "persistent stage launches (batches) "
                            "(hit_solver_b200.autotune)", **tuning},
        "gpu_launches": K * launches_per_step,
        "clocks": clk.summary(),
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    return line


def hit_forms(K: int, W: int, B: int, flush, world: int):
    """512^2 production forced HIT (device forcing noise): the plain FP64
    single solve and B FP32-bulk solves (seeds 0..B-1, Mach 0.1..0.4) in one
    batch, both device-timed with L2 flushes."""
    import torch

    from hit_solver_b200 import _lib
    from hit_solver_b200.batch import Batch
    from hit_solver_b200.hit2d import HITSolver
    from hit_solver_b200.serving import hit_request_config

    n = NX
    from hit_solver_b200 import autotune

    s64 = HITSolver(hit_request_config(n, 1234, 0.25, 10 ** 9, "fp64"))
    t64 = autotune.tune_plan(s64.plan, s64.q)
    s64.advance(W)
    k64 = max(K // 2, 5)
    tune64 = t64
    t64 = dist_max(timed_steps(lambda: s64.advance(1), k64, flush), world)
    del s64
    solvers = [HITSolver(hit_request_config(n, i, 0.1 + 0.3 * i / max(B - 1, 1), 10 ** 9,
                                            "fp32-bulk")) for i in range(B)]
    batch = Batch.from_plans([s.plan for s in solvers], [s.q for s in solvers])
    tuneb = batch.autotune()
    batch.run(W)
    kb = max(K // 4, 5)
    tb = dist_max(timed_steps(lambda: batch.run(1), kb, flush), world)
    status = max(int(m.scalars()[_lib.S_STATUS]) for m in batch.members)
    batch.close()
    del solvers
    torch.cuda.synchronize()
    plain = world * n * n * k64 / t64
    batched = world * B * n * n * kb / tb
    return {"workload": "hit_production_512x512 (nu 7.5e-4, OU 3..5, Mach control, drag, cooling)",
            "plain_fp64": {"value": plain, "ms_per_step": 1e3 * t64 / k64},
            "batched_fp32": {"value": batched, "ms_per_step": 1e3 * tb / kb, "solves": B},
            "speedup_batched_vs_plain": batched / plain, "status_bits": status,
            "_tuning": {"plain_fp64": tune64, "batched_fp32": tuneb}}


def ensemble_run(K: int, W: int, flush, world: int, count: int):
    """The batched-ensemble configuration: `count` production-physics HIT
    solves with grids drawn from {128, 256, 384, 512}^2, seeds 0..count-1 and
    turbulent Mach uniform in [0.1, 0.4] (fixed meta-seed), FP32-bulk, one
    launch per kernel of the step for all of them, autotuned."""
    import numpy as np
    import torch

    from hit_solver_b200.batch import Batch
    from hit_solver_b200.hit2d import HITSolver
    from hit_solver_b200.serving import hit_request_config

    rng = np.random.default_rng(64)
    sizes = rng.choice([128, 256, 384, 512], size=count)
    machs = rng.uniform(0.1, 0.4, size=count)
    solvers = [HITSolver(hit_request_config(int(n), i, float(m), 10 ** 9, "fp32-bulk"))
               for i, (n, m) in enumerate(zip(sizes, machs))]
    batch = Batch.from_plans([s.plan for s in solvers], [s.q for s in solvers])
    knobs = batch.autotune()
    batch.run(W)
    k = max(K // 8, 5)
    t = dist_max(timed_steps(lambda: batch.run(1), k, flush), world)
    from hit_solver_b200 import _lib

    status = max(int(m.scalars()[_lib.S_STATUS]) for m in batch.members)
    cells = int(sum(int(n) * int(n) for n in sizes))
    batch.close()
    del solvers
    torch.cuda.synchronize()
    return {"workload": f"{count} HIT solves, grids from {{128,256,384,512}}^2, Mach U[0.1,0.4]",
            "value": world * cells * k / t, "unit": "cell-updates/s", "ms_per_step": 1e3 * t / k,
            "cells": cells, "solves": count, "steps": k, "tuning": knobs, "status_bits": status}


def spectra_run(K: int, W: int, flush, world: int, count: int, cpu: bool):
    """Shell spectra (the per-snapshot work of HIT2DSpectra.compute) of `count`
    device-resident 512^2 snapshots per step: fluctuation fields (CUDA),
    rfft2 of the four fields (the library's own line transforms), shell
    binning (CUDA).  Phase times come from CUDA events around each call of a
    separate pass; cuFFT's rfft2 of the same fields is timed beside it as a
    comparison."""
    import numpy as np
    import torch

    from hit_solver_b200 import _lib, core
    from hit_solver_b200.postprocess import shell_spectra

    gen = torch.Generator(device="cuda").manual_seed(5)
    shape = (count, NY, NX)
    rho = 1.0 + 0.3 * torch.rand(shape, generator=gen, device="cuda", dtype=torch.float64)
    u = 0.2 * torch.randn(shape, generator=gen, device="cuda", dtype=torch.float64)
    v = 0.2 * torch.randn(shape, generator=gen, device="cuda", dtype=torch.float64)
    h = 2.0 * math.pi / NX
    run = lambda: shell_spectra(rho, u, v, h, h, "reynolds")  # noqa: E731
    for _ in range(W):
        run()
    k = max(K // 20, 5)
    t = dist_max(timed_steps(run, k, flush), world)
    # phase times: the same three calls with events between them
    lib = _lib.load()
    nh = NX // 2 + 1
    ns = min(NX, NY) // 2 + 1
    ws = torch.empty(int(lib.hitb200_spectra_workspace_bytes(count, NX, NY)), dtype=torch.uint8,
                     device="cuda")
    fields = torch.empty((count, 4, NY, NX), dtype=torch.float64, device="cuda")
    e = torch.empty((count, ns), dtype=torch.float64, device="cuda")
    z = torch.empty_like(e)
    st = torch.cuda.current_stream()
    ph = {"fields": 0.0, "rfft2": 0.0, "shells": 0.0}
    spec = torch.empty((count, 4, NY, nh), dtype=torch.complex128, device="cuda")
    fws = torch.empty(int(lib.hitb200_rfft2_workspace_bytes(NX, NY)), dtype=torch.uint8, device="cuda")
    cufft_ms = 0.0
    torch.fft.rfft2(fields)  # the library's plan, built once outside the timing
    torch.cuda.synchronize()
    for _ in range(k):
        flush.zero_()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(st)
        _lib.check(lib.hitb200_spectra_fields(rho.data_ptr(), u.data_ptr(), v.data_ptr(), count, NX,
                                              NY, 0, fields.data_ptr(), ws.data_ptr(), ws.numel(),
                                              core.stream_handle()))
        ev[1].record(st)
        _lib.check(lib.hitb200_rfft2(fields.data_ptr(), 4 * count, NX, NY, spec.data_ptr(),
                                     fws.data_ptr(), fws.numel(), core.stream_handle()))
        ev[2].record(st)
        _lib.check(lib.hitb200_spectra_shells(spec.data_ptr(), count, NX, NY, h, h, e.data_ptr(),
                                              z.data_ptr(), ws.data_ptr(), ws.numel(),
                                              core.stream_handle()))
        ev[3].record(st)
        torch.cuda.synchronize()
        for i, name in enumerate(ph):
            ph[name] += ev[i].elapsed_time(ev[i + 1]) / k
        # comparison: the library FFT (cuFFT) on the same fields
        flush.zero_()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(st)
        ref = torch.fft.rfft2(fields)
        c1.record(st)
        torch.cuda.synchronize()
        cufft_ms += c0.elapsed_time(c1) / k
        del ref
    peak, _kind = measured_peak()
    cells = count * NX * NY
    # algorithmic bytes: fields = mean pass (read rho, u, v) + field pass (read
    # rho, u, v, write 4 fields); shells = read the 4 half spectra (16 B a mode)
    fbytes = cells * (24 + 24 + 32)
    sbytes = count * 4 * NY * nh * 16
    phases = {
        "fields": {"ms": ph["fields"], "gbs": fbytes / (ph["fields"] / 1e3) / 1e9,
                   "bytes": fbytes, "frac": fbytes / (ph["fields"] / 1e3) / 1e9 / peak},
        "rfft2": {"ms": ph["rfft2"], "impl": "hitb200_rfft2 (the library's line transforms: radix-8 in registers for power-of-two lengths)",
                  "cufft_ms": cufft_ms},
        "shells": {"ms": ph["shells"], "gbs": sbytes / (ph["shells"] / 1e3) / 1e9, "bytes": sbytes,
                   "frac": sbytes / (ph["shells"] / 1e3) / 1e9 / peak},
    }
    out = {"workload": f"shell spectra of {count} resident {NX}x{NY} snapshots (Reynolds)",
           "value": world * count * k / t, "unit": "snapshots/s", "ms_per_step": 1e3 * t / k,
           "snapshots": count, "steps": k, "phases": phases,
           "l2": "flushed (320 MB write) before every timed step"}
    if cpu:
        from oracle import spectra_oracle as SO

        x = (np.arange(NX) + 0.5) * h
        r0, u0, v0 = (a[0].cpu().numpy() for a in (rho, u, v))
        SO.snapshot_shells(x, x, r0, u0, v0, "reynolds")
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            SO.snapshot_shells(x, x, r0, u0, v0, "reynolds")
        tc = (time.perf_counter() - t0) / reps
        out["cpu_baseline"] = {"value": 1.0 / tc, "unit": "snapshots/s", "cores": 1, "kind": "port",
                               "sample": f"{reps} snapshots of {NX}x{NY} through the NumPy oracle"}
    del rho, u, v, fields, ws
    torch.cuda.synchronize()
    return out


def initial_state_run(n: int = 1024, reps: int = 5):
    """Building one n^2 initial state, the host form (NumPy, the reference's
    arithmetic) against the device form (CUDA kernels, own line transforms): the
    admission cost of a solve."""
    import numpy as np
    import torch

    from hit_solver_b200.hit2d import (HIT2DConfig, create_grid, initialize_hit_2d,
                                       initialize_hit_2d_device)
    from hit_solver_b200.equations import EulerEquation2D
    from hit_solver_b200.problems.riemann import RiemannConfig3

    cfg = HIT2DConfig(nx=n, ny=n, target_mach=0.25, initial_kmin=3, initial_kmax=5)
    dom = create_grid(cfg)[0]
    eq = EulerEquation2D(gamma=cfg.gamma)

    def clock(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return 1e3 * (time.perf_counter() - t0) / reps

    rc = RiemannConfig3(nx=n, ny=n)
    return {
        "workload": f"one {n}x{n} initial state: wall time, host form incl. its upload",
        "hit_host_ms": clock(lambda: initialize_hit_2d(cfg, dom, eq, np.random.default_rng(1))),
        "hit_device_ms": clock(lambda: initialize_hit_2d_device(cfg, dom, eq, np.random.default_rng(1))),
        "riemann_device_ms": clock(rc.initial_state),
    }


def dropin_hit_run(steps: int = 50):
    """The drop-in HIT path (what ``run_hit2d.py --backend b200`` runs): the
    mirror's HITSolver on the 512^2 production physics with the reference's
    NumPy forcing-noise stream, continued on the device (``numpy``, graph
    replay) and drawn by NumPy on the host and uploaded each step
    (``numpy-host``); device-timed per step.  Plus the mirror's
    run_simulation for the same physics end to end (60 steps, diagnostics and
    snapshots only at the ends, host wall clock including its setup)."""
    import tempfile

    import torch

    from hit_solver_b200.hit2d import HIT2DConfig, HITSolver, run_simulation

    kw = dict(nx=NX, ny=NY, tfinal=1e9, cfl=0.05, target_mach=0.25, initial_kmin=3,
              initial_kmax=5, forcing_kmin=3.0, forcing_kmax=5.0, forcing_correlation_time=0.5,
              mach_control=True, mach_control_target=0.25, viscosity=7.5e-4,
              hyperviscosity_mn=0.002, large_scale_drag=0.10, cooling_time=5.0, precision="fp64")
    out = {"workload": "hit_production_512x512, reference NumPy noise stream, FP64"}
    st = torch.cuda.current_stream()
    for mode, k in (("numpy", steps), ("numpy-host", max(steps // 5, 5))):
        s = HITSolver(HIT2DConfig(forcing_noise=mode, **kw))
        s.advance(3)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        s.advance(k)
        b.record(st)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / k
        out[mode] = {"ms_per_step": ms, "value": NX * NY / (ms / 1e3), "unit": "cell-updates/s",
                     "steps": k}
        del s
    out["speedup_device_stream"] = out["numpy-host"]["ms_per_step"] / out["numpy"]["ms_per_step"]
    with tempfile.TemporaryDirectory() as tmp:
        cfg = HIT2DConfig(forcing_noise="numpy", max_steps=60, diagnostics_every=10 ** 6,
                          snapshot_every=10 ** 6, output_dir=Path(tmp), **kw)
        import contextlib
        import io

        t0 = time.perf_counter()
        with contextlib.redirect_stdout(io.StringIO()):
            run_simulation(cfg)
        torch.cuda.synchronize()
        out["run_simulation_60_steps_s"] = time.perf_counter() - t0
    return out


def serving_run(args):
    """Continuous batching of a seeded Poisson stream (Riemann config 3/6 on
    256..1024^2 to tfinal, HIT 128..512^2 for 200 steps), served three times;
    p50/p99 of each repeat and their medians, the host time of each phase of
    the loop, and the solo time of the request with the longest latency (its
    lower bound on an idle GPU)."""
    import statistics

    import torch

    from hit_solver_b200 import serving

    reqs = serving.poisson_requests(args.serve_requests, args.serve_rate, seed=2024)
    reps = []
    for _ in range(3):
        server = serving.SolveServer("fp32-bulk", steps_per_round=args.serve_round)
        results = server.serve(reqs)
        torch.cuda.synchronize()
        reps.append((dict(server.stats), results))
    st = dict(reps[-1][0])
    st["p50_s"] = statistics.median(r[0]["p50_s"] for r in reps)
    st["p99_s"] = statistics.median(r[0]["p99_s"] for r in reps)
    st["cell_updates_per_s"] = statistics.median(r[0]["cell_updates_per_s"] for r in reps)
    st["repeats"] = [{k: round(r[0][k], 4) for k in ("p50_s", "p99_s", "makespan_s", "admit_s",
                                                      "rebuild_s", "round_s")} for r in reps]
    slowest = max(reps[-1][1], key=lambda r: r.latency)
    req = next(r for r in reqs if r.rid == slowest.rid)
    t0 = time.perf_counter()
    serving.run_alone(req)
    torch.cuda.synchronize()
    st["slowest_request"] = {"kind": req.kind, "n": req.n, "steps": slowest.steps,
                             "latency_s": round(slowest.latency, 4),
                             "solo_s": round(time.perf_counter() - t0, 4)}
    st.update({"rate_per_s": args.serve_rate, "unit": "cell-updates/s",
               "mix": {k: sum(1 for r in reqs if r.kind == k) for k in serving.KINDS},
               "failed": sum(1 for r in reps[-1][1] if r.status != 0)})
    return st


def cpu_baseline(steps: int):
    """The oracle (NumPy FP64 port of the reference algorithm) on `steps` RK3
    steps of the same 512^2 workload, one process."""
    import numpy as np

    from oracle import hit_oracle as O

    prm = O.RiemannParams(number=3, nx=NX, ny=NY)
    q, dt, n = O.riemann_setup(prm)
    O.riemann_run(prm, max_steps=1, q0=q, dt=dt)  # warm-up
    t0 = time.perf_counter()
    O.riemann_run(prm, max_steps=steps, q0=q, dt=dt)
    el = time.perf_counter() - t0
    return {"value": NX * NY * steps / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"{steps} RK3 steps of the 512x512 workload, NumPy FP64 oracle, 1 process "
                      f"({el:.1f} s)"}


# ----------------------------------------------------------------------------------
# reference arm: the reference algorithm's CPU implementation on all host cores
# ----------------------------------------------------------------------------------
def _ref_worker(args):
    steps, seed = args
    import numpy as np

    from oracle import hit_oracle as O

    prm = O.RiemannParams(number=3, nx=NX, ny=NY)
    q, dt, n = O.riemann_setup(prm)
    O.riemann_run(prm, max_steps=1, q0=q, dt=dt)
    t0 = time.perf_counter()
    O.riemann_run(prm, max_steps=steps, q0=q, dt=dt)
    return time.perf_counter() - t0


def run_reference(args, world, rank):
    if rank != 0:
        return None
    import multiprocessing as mp

    os.environ.setdefault("OMP_NUM_THREADS", "1")
    cores = os.cpu_count() or 1
    procs = max(1, min(cores, 32))  # each process holds ~0.5 GB of NumPy temporaries
    if args.ref_procs > 0:
        procs = min(procs, args.ref_procs)
    # bounded sample: each process advances the 512^2 workload a few steps;
    # ~4 s per step per process, so the run stays within a few minutes
    steps = max(1, min(args.steps, 8))
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        times = pool.map(_ref_worker, [(steps, i) for i in range(procs)])
    wall = time.perf_counter() - t0
    slowest = max(times)
    value = procs * NX * NY * steps / slowest
    return {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": steps, "warmup": 1, "ms_per_step": 1e3 * slowest / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
        "data": "synthetic: the reference's own Riemann config-3 initial state",
        "config": {**WORKLOAD, "precision": "fp64", "parallelism": f"{procs} host processes"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": procs, "kind": "port",
                         "sample": f"{steps} RK3 steps of the 512x512 workload in each of {procs} "
                                   f"processes (NumPy FP64 oracle; wall {wall:.1f} s)"},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            line = run_reference(args, world, rank)
        else:
            line = run_b200(args, world, rank, local)
        if rank == 0 and line is not None:
            print(json.dumps(line))
    finally:
        dist_finish(world)


if __name__ == "__main__":
    main()
