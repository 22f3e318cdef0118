"""The forcing-noise stream of the reference reproduced from its definition.

The reference draws its OU forcing noise as
``np.random.default_rng(seed).standard_normal((ny, nx))`` once per step
(OOP/forcing.py:66,77).  The device generator (noise_mode 2) restates that
stream: PCG64 (128-bit LCG, XSL-RR output) and NumPy's 256-level ziggurat
with the table in hit_solver_b200/csrc/ziggurat_table.inc.  Here a plain
Python restatement of the same sampler over the committed table is checked
draw for draw against NumPy itself, for several seeds, so that the table and
the algorithm the CUDA kernels implement are pinned on the CPU; the GPU test
checks the kernels against NumPy field for field.
"""

import math
import re
from pathlib import Path

import numpy as np
import pytest

INC = Path(__file__).resolve().parent.parent / "hit_solver_b200" / "csrc" / "ziggurat_table.inc"
PCG_MULT = (2549297995355413924 << 64) + 4865540595714422341
MASK128 = (1 << 128) - 1
R0 = 3.6541528853610088


def load_table():
    text = INC.read_text()

    def arr(name, conv):
        body = re.search(name + r"\[256\] = \{(.*?)\};", text, re.S).group(1)
        return [conv(t.strip().rstrip("ull")) for t in body.split(",")]

    return arr("kZigW", float), arr("kZigK", int), arr("kZigF", float)


def pcg64_raw(state: int, inc: int, n: int):
    out = []
    for _ in range(n):
        state = (state * PCG_MULT + inc) & MASK128
        hi, lo = state >> 64, state & ((1 << 64) - 1)
        x, rot = hi ^ lo, state >> 122
        out.append(((x >> rot) | (x << (64 - rot))) & ((1 << 64) - 1))
    return out, state


def normals(raws, n, w, k, f):
    out, pos = [], 0

    def nd():
        nonlocal pos
        v = raws[pos]
        pos += 1
        return (v >> 11) * (1.0 / 9007199254740992.0)

    inv_r = 1.0 / R0
    while len(out) < n:
        r = raws[pos]
        pos += 1
        idx = r & 0xFF
        r >>= 8
        sign = r & 1
        rabs = (r >> 1) & 0x000FFFFFFFFFFFFF
        x = rabs * w[idx]
        if sign:
            x = -x
        if rabs < k[idx]:
            out.append(x)
            continue
        if idx == 0:
            while True:
                xx = -inv_r * math.log1p(-nd())
                yy = -math.log1p(-nd())
                if yy + yy > xx * xx:
                    out.append(-(R0 + xx) if (rabs >> 8) & 1 else R0 + xx)
                    break
            continue
        if (f[idx - 1] - f[idx]) * nd() + f[idx] < math.exp(-0.5 * x * x):
            out.append(x)
    return np.array(out), pos


def test_pcg64_restatement_matches_numpy():
    g = np.random.PCG64(1235)
    st = g.state["state"]
    mine, _ = pcg64_raw(st["state"], st["inc"], 1000)
    assert mine == g.random_raw(1000).tolist()


@pytest.mark.parametrize("seed", [1235, 7, 2 ** 31 - 1])
def test_ziggurat_table_reproduces_numpy_normals(seed):
    w, k, f = load_table()
    n = 400_000
    want = np.random.default_rng(seed).standard_normal(n)
    raws = np.random.PCG64(seed).random_raw(n + n // 8).tolist()
    got, used = normals(raws, n, w, k, f)
    np.testing.assert_array_equal(got, want)
    # the stream continues where NumPy's does
    g = np.random.default_rng(seed)
    g.standard_normal(n)
    ref = np.random.PCG64(seed)
    ref.advance(used)
    assert g.bit_generator.state["state"] == ref.state["state"]


@pytest.mark.gpu
@pytest.mark.parametrize("ny,nx,seed", [(512, 512, 1235), (96, 80, 7), (33, 1000, 2 ** 31 - 1)])
def test_device_stream_matches_numpy(ny, nx, seed):
    """Three consecutive standard_normal((ny, nx)) fields of the device stream
    (hitb200_noise_field) against NumPy's, and the stream position after them.
    Draws on the ziggurat's tail use CUDA's log1p, so a tail normal may differ
    from NumPy's in its last bits; everything else is bit for bit."""
    import torch

    from hit_solver_b200 import _lib, core
    from hit_solver_b200.hit2d import HIT2DConfig, create_grid, hit_descriptor

    cfg = HIT2DConfig(nx=nx, ny=ny, forcing_kmin=1.0, forcing_kmax=3.0, forcing_noise="numpy")
    plan = core.Plan(hit_descriptor(cfg, create_grid(cfg)[0]))
    rng = np.random.default_rng(seed)
    plan.set_noise_stream(rng.bit_generator.state)
    out = torch.empty((ny, nx), dtype=torch.float64, device="cuda")
    for _ in range(3):
        _lib.check(plan.lib.hitb200_noise_field(plan.handle, out.data_ptr(), core.stream_handle()))
        got = out.cpu().numpy()
        want = rng.standard_normal((ny, nx))
        diff = got != want
        # only tail draws (|x| > r0) may differ, and by roundoff
        assert np.all(np.abs(want[diff]) > R0), np.abs(want[diff]).min() if diff.any() else None
        assert np.all(np.abs(got[diff] - want[diff]) <= 1e-14 * np.abs(want[diff]))
        assert diff.sum() <= max(4, 1e-3 * ny * nx)
    assert plan.noise_stream()["state"] == rng.bit_generator.state["state"]
