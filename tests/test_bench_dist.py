"""The multi-process plumbing of bench.py on CPU (gloo, world size 2).

A solve does not shard, so bench.py --gpus N runs one replica per rank; the
only cross-rank steps are barriers and the max-over-ranks timing.  These
tests run that plumbing with two gloo ranks on the host, and the reference
arm under torchrun with two ranks (rank 0 measures and prints one JSON line,
rank 1 exits cleanly without work).
"""

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as tmp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    bench.dist_barrier(world)
    out[rank] = bench.dist_max(1.5 + rank, world)
    bench.dist_barrier(world)
    bench.dist_finish(world)


def test_dist_max_over_two_gloo_ranks():
    port = _free_port()
    out = tmp.Manager().dict()
    tmp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
    assert dict(out) == {0: 2.5, 1: 2.5}


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--ref-procs", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    res = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
