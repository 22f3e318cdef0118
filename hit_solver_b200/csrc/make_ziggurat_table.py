"""Generate ``ziggurat_table.inc``: the 256-level ziggurat of NumPy's
``Generator.standard_normal`` (the forcing noise of OOP/forcing.py:66,77 is
``np.random.default_rng(seed).standard_normal((ny, nx))``).

    python hit_solver_b200/csrc/make_ziggurat_table.py

NumPy (BSD-3; 2.x, in use here) draws a normal from one 64-bit PCG64 output
r: idx = r & 0xff, sign = bit 8, rabs = the next 52 bits; x = +-rabs *
w[idx] is returned when rabs < k[idx] (Marsaglia and Tsang, "The Ziggurat
Method for Generating Random Variables", J. Stat. Softw. 5(8), 2000; 256
levels of area v, base strip at r_0 = 3.6541528853610088), else the wedge or
tail test decides with further uniforms.  The tables follow from that
construction:

    x_255 = r_0,  x_{i-1} = sqrt(-2 log(v / x_i + f(x_i))),  f(x) = exp(-x^2 / 2)
    w_i = x_i / 2^52,  w_0 = (v / f(r_0)) / 2^52,  k_i = floor(x_{i-1} / x_i 2^52),
    k_0 = floor(r_0 f(r_0) / v 2^52),  k_1 = 0,  f_i = f(x_i),  f_0 = 1

with v = 0.004928673233974652.  Evaluated in double precision this
reproduces NumPy's w exactly for levels 0 and 38..255; the top levels 1..37,
where the recursion amplifies rounding, differ from NumPy's values by up to
22 ulp.  Their exact values are therefore pinned here from NumPy's own
draws: for each level, every accepted sample x = rabs * w bounds w to an
interval of reals, and a single double lies in the intersection.  k and f of
those levels then follow from the pinned x by the formulas above.  The
committed table is checked draw for draw against NumPy by
tests/test_numpy_noise.py.
"""

from __future__ import annotations

import math
from fractions import Fraction
from pathlib import Path

import numpy as np

R0 = 3.6541528853610088
V = 0.004928673233974652
M52 = 2.0 ** 52
PIN_TOP = 37  # levels 1..PIN_TOP are pinned from NumPy's draws
OUT = Path(__file__).resolve().parent / "ziggurat_table.inc"


def recursion():
    f = lambda x: math.exp(-0.5 * x * x)
    x = [0.0] * 256
    x[255] = R0
    for i in range(254, 0, -1):
        x[i] = math.sqrt(-2.0 * math.log(V / x[i + 1] + f(x[i + 1])))
    w = [0.0] * 256
    w[0] = (V / f(R0)) / M52
    for i in range(1, 256):
        w[i] = x[i] / M52
    return w


def tables(w):
    f = lambda x: math.exp(-0.5 * x * x)
    x = [wi * M52 for wi in w]  # exact: division by a power of two
    k = [0] * 256
    fi = [0.0] * 256
    k[0] = int(R0 * f(R0) / V * M52)
    k[1] = 0
    for i in range(2, 256):
        k[i] = int(x[i - 1] / x[i] * M52)
    fi[0] = 1.0
    for i in range(1, 256):
        fi[i] = f(x[i])
    return k, fi


def _raw_normals(raws, want, w, k, fi, level_samples):
    """Walk NumPy's draws with the candidate tables (their fast / wedge / tail
    decisions), collecting (rabs, |x|) of every accepted non-tail sample per
    level."""
    pos = 0
    inv_r = 1.0 / R0

    def nd():
        nonlocal pos
        v = raws[pos]
        pos += 1
        return (v >> 11) * (1.0 / 9007199254740992.0)

    n = 0
    while n < len(want):
        rr = raws[pos]
        pos += 1
        idx = rr & 0xFF
        rr >>= 8
        rabs = (rr >> 1) & 0x000FFFFFFFFFFFFF
        x = rabs * w[idx]
        if rabs < k[idx]:
            level_samples[idx].append((rabs, abs(float(want[n]))))
            n += 1
            continue
        if idx == 0:
            while True:
                xx = -inv_r * math.log1p(-nd())
                yy = -math.log1p(-nd())
                if yy + yy > xx * xx:
                    n += 1
                    break
            continue
        if (fi[idx - 1] - fi[idx]) * nd() + fi[idx] < math.exp(-0.5 * x * x):
            level_samples[idx].append((rabs, abs(float(want[n]))))
            n += 1


def pin(w, k, fi, draws=3_000_000, seed=7):
    want = np.random.default_rng(seed).standard_normal(draws)
    raws = np.random.PCG64(seed).random_raw(2 * draws).tolist()
    samples = [[] for _ in range(256)]
    _raw_normals(raws, want, w, k, fi, samples)
    pinned = list(w)
    for i in range(1, PIN_TOP + 1):
        s = samples[i][:200]
        lo = max((Fraction(ax) - Fraction(math.ulp(ax)) / 2) / r for r, ax in s)
        hi = min((Fraction(ax) + Fraction(math.ulp(ax)) / 2) / r for r, ax in s)
        c = math.nextafter(float(lo), -math.inf)
        cands = []
        for _ in range(8):
            if lo <= Fraction(c) <= hi and all(r * c == ax for r, ax in s):
                cands.append(c)
            c = math.nextafter(c, math.inf)
        if len(cands) != 1:
            raise RuntimeError(f"level {i}: {len(cands)} candidate widths")
        pinned[i] = cands[0]
    return pinned


def main():
    w = recursion()
    k, fi = tables(w)
    w = pin(w, k, fi)
    k, fi = tables(w)
    with OUT.open("w") as fh:
        fh.write("// Generated by make_ziggurat_table.py: NumPy's standard_normal ziggurat\n")
        fh.write("// (256 levels; w = widths / 2^52, k = fast-path bounds, f = exp(-x^2 / 2)).\n")
        fh.write("static const double kZigW[256] = {\n")
        fh.write(",\n".join(f"    {v!r}" for v in w) + "};\n")
        fh.write("static const unsigned long long kZigK[256] = {\n")
        fh.write(",\n".join(f"    {v}ull" for v in k) + "};\n")
        fh.write("static const double kZigF[256] = {\n")
        fh.write(",\n".join(f"    {v!r}" for v in fi) + "};\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
