"""Generates tests/golden/golden_modes.npz: known answers for the two
reference modes beside the canonical one, from their independent Python
statements (tests/test_compat_restatement.py: the reference's default
square-region, scaled-lattice, z-code rules; tests/test_spacetime_restatement.py:
the space-time rules with lifted time distances), which share no code with
the C oracle or the CUDA engine.  Small seeded cases with repeated
positions (ties) and origins away from zero.

Run:  python tests/golden/make_golden_modes.py
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))                       # tests/

from test_compat_restatement import compat_restated              # noqa: E402
from test_spacetime_restatement import spacetime_restated        # noqa: E402

OUT = os.path.join(HERE, "golden_modes.npz")


def z_multiplier(sr, scale, cell, zmax, pmin):
    # terranni.cpp:675-684
    pw = int(math.ceil(2.0 * sr * scale / cell))
    max_sum = pw * pw * (zmax - pmin)
    m = 1
    if max_sum < 2147483647:
        m = int(math.floor(2147483647 / max_sum))
        m = int(10 ** math.floor(math.log10(m)))
    return m


def main():
    out = {}
    compat_cases = [
        (5, 2.0, 5.0, 4.99, 0, 8, 6, (0.0, 0.0), 50),
        (3, 1.0, 3.0, 2.5, -4, 9, 7, (250.0, -125.0), 45),
        (1, 2.0, 6.0, 5.0, 10, 10, 8, (500100.0, 4100200.0), 30),
    ]
    for k, (scale, cell, sr, qr, pmin, ncols, nrows, origin, n) in enumerate(compat_cases):
        rng = np.random.default_rng(1000 + k)
        pts = np.stack([origin[0] + rng.uniform(-2, ncols * cell + 2, n),
                        origin[1] + rng.uniform(-2, nrows * cell + 2, n), rng.uniform(12, 48, n)], 1)
        pts = np.concatenate([pts, pts[:6]])
        pts[-6:, 2] += 3.0
        mult = z_multiplier(sr, scale, cell, float(pts[:, 2].max()), pmin)
        h, res = compat_restated(scale, cell, sr, qr, pmin, mult, origin[0], origin[1], nrows, ncols, pts)
        p = f"compat{k}_"
        out[p + "params"] = np.array([scale, cell, sr, qr, pmin, mult, origin[0], origin[1], nrows, ncols],
                                     np.float64)
        out[p + "pts"], out[p + "h"], out[p + "res"] = pts, h, res
    # near-ties: pairs of sites mirrored about pixel centres, at UTM-scale
    # origins, where the depth test is decided by the last bits of the planes;
    # with drawPlane's double-then-round slopes (nni.cpp:194-200) the kept
    # site differs in some cells from a rule that rounds the site offset to
    # float first
    for m, seed in enumerate((6, 8)):
        k = len(compat_cases) + m
        rng = np.random.default_rng(seed)
        scale, cell, sr, qr, pmin, ncols, nrows = 1, 1.0, 3.0, 2.5, 0, 5, 5
        origin = (500000.0 + float(rng.integers(0, 1000)) + 0.25, 4100000.0 + float(rng.integers(0, 1000)) + 0.5)
        ps = cell / scale
        po = math.ceil((float(np.float32(qr)) - math.floor(scale / 2.0) * ps) / ps) + 1
        left = 0 - cell / 2.0 - po * ps
        pts = []
        for _ in range(12):
            pi = int(rng.integers(0, ncols * scale + 2 * po))
            pj = int(rng.integers(0, nrows * scale + 2 * po))
            cx, cy = left + (pi + 0.5) * ps, left + (pj + 0.5) * ps
            d, ang = rng.uniform(0.2, 0.6), rng.uniform(0, math.pi)
            ex, ey = d * math.cos(ang), d * math.sin(ang)
            z1, z2 = rng.uniform(10, 40, 2)
            pts.append((origin[0] + cx + ex, origin[1] + cy + ey, z1))
            pts.append((origin[0] + cx - ex, origin[1] + cy - ey, z2))
        pts = np.array(pts)
        mult = 1000
        h, res = compat_restated(scale, cell, sr, qr, pmin, mult, origin[0], origin[1], nrows, ncols, pts)
        p = f"compat{k}_"
        out[p + "params"] = np.array([scale, cell, sr, qr, pmin, mult, origin[0], origin[1], nrows, ncols],
                                     np.float64)
        out[p + "pts"], out[p + "h"], out[p + "res"] = pts, h, res
    st_cases = [
        (8, 6, 100, (-2, -1, 10, 8), 5, 1, 100, 40),
        (7, 7, 50, (0, 0, 7, 7), -2, 2, 40, 36),
        (6, 5, 100, (-1, -1, 7, 6), 0, 3, 250, 30),
    ]
    for k, (ncols, nrows, cs, raster, cur, rt, tau, n) in enumerate(st_cases):
        rng = np.random.default_rng(2000 + k)
        xyz = np.stack([rng.integers(-2 * cs, (ncols + 2) * cs, n), rng.integers(-2 * cs, (nrows + 2) * cs, n),
                        rng.integers(-500, 500, n)], 1).astype(np.int32)
        t = rng.integers(cur - 3 * rt - 1, cur + 3 * rt + 2, n).astype(np.int32)
        xyz[3, :2] = xyz[2, :2]
        t[3] = t[2]
        Z, C, h = spacetime_restated(ncols, nrows, cs, raster, xyz, t, cur, rt, tau)
        p = f"st{k}_"
        out[p + "params"] = np.array([ncols, nrows, cs, *raster, cur, rt, tau], np.int64)
        out[p + "xyz"], out[p + "t"], out[p + "Z"], out[p + "C"], out[p + "h"] = xyz, t, Z, C, h
    out["n_compat"] = np.array([len(compat_cases) + 2])
    out["n_st"] = np.array([len(st_cases)])
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
