"""A second, independent statement of the space-time rules for tiny cases in
plain Python integers: per slice the lifted-nearest site of every raster
pixel by brute force, then every grid cell tested directly against every
pixel's disc (no row spans).  oracle.interpolate_spacetime must agree on Z
and C exactly and on the heights bit for bit."""
import numpy as np
import pytest


def spacetime_restated(ncols, nrows, cs, raster, xyz, t, cur, rt, tau, z_scale=0.01, z_offset=0.0):
    rx0, ry0, rx1, ry1 = raster
    ex = max(rx1, ncols) - min(rx0, 0)
    ey = max(ry1, nrows) - min(ry0, 0)
    cap = ex * ex + ey * ey
    Z = [[0] * ncols for _ in range(nrows)]
    C = [[0] * ncols for _ in range(nrows)]
    pts = [(int(x), int(y), int(z), int(tt), k) for k, ((x, y, z), tt) in enumerate(zip(xyz.tolist(), t.tolist()))]
    for j in range(-rt, rt + 1):
        ts = cur + j
        sites = [p for p in pts if abs(ts - p[3]) <= rt]
        for py in range(ry0, ry1):
            for px in range(rx0, rx1):
                best = None
                for (x, y, z, tt, k) in sites:
                    d = (x - px * cs) ** 2 + (y - py * cs) ** 2 + ((ts - tt) * tau) ** 2
                    key = (d, k, z)
                    if best is None or key < best:
                        best = key
                if best is None:
                    continue
                e = best[0] - (j * tau) ** 2
                if e < 0:
                    continue
                R2 = min(e // (cs * cs), cap)
                for qy in range(nrows):
                    for qx in range(ncols):
                        if (qx - px) ** 2 + (qy - py) ** 2 <= R2:
                            Z[qy][qx] += best[2]
                            C[qy][qx] += 1
    Z, C = np.array(Z, np.int64), np.array(C, np.int64)
    h = np.where(C > 0, (Z / np.maximum(C, 1)) * z_scale + z_offset, -9999.0).astype(np.float32)
    return Z, C, h


@pytest.mark.parametrize("rt,tau,raster", [(1, 100, (-2, -1, 9, 8)), (2, 37, (0, 0, 7, 6)), (0, 100, (-1, -1, 8, 7))])
def test_spacetime_oracle_matches_an_independent_restatement(oracle, rt, tau, raster):
    rng = np.random.default_rng(rt * 10 + tau)
    n = 40
    xyz = np.stack([rng.integers(-250, 950, n), rng.integers(-250, 850, n), rng.integers(-500, 500, n)], 1)
    xyz[3, :2] = xyz[2, :2]                               # a tie on position
    t = rng.integers(5 - 3 * rt - 1, 5 + 3 * rt + 2, n)
    t[3] = t[2]
    wp = oracle.make_wp(7, 6, 100, raster=raster)
    r = oracle.interpolate_spacetime(wp, xyz.astype(np.int32), t.astype(np.int32), 5, rt, tau)
    Z, C, h = spacetime_restated(7, 6, 100, raster, xyz, t, 5, rt, tau)
    assert np.array_equal(r["Z"], Z) and np.array_equal(r["C"], C)
    assert np.array_equal(r["h"].view(np.uint32), h.view(np.uint32))
