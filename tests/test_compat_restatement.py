"""A second, independent statement of the reference-default rules
(nni.cpp:171-230 drawPlane, 483-549 queries and z-codes, 733-737 LEQUAL,
803-807 the query depth test, 836-848 dequantisation, cuda_nni.cu:423-503
int32 sums and truncating divide, nni.cpp:879-886 the raster), written as
plain loops over numpy float32 and Python float (double) scalars for tiny
cases, one rounding per operation in the formulas' order.  The oracle's C
restatement (oracle.compat) must agree with it bit for bit; the GPU is then
checked against the oracle (tests/test_gpu_compat.py)."""
import math

import numpy as np
import pytest

F = np.float32


def _plane(hw, dx, dy):
    """drawPlane's slopes and offset (nni.cpp:186-200): zpx, zpy, a and b
    are formed in double from the double site offset and rounded to float
    once each; the offset is a float sum of float squares."""
    h = float(hw)
    zpx = F((dx + h) / h)
    zpy = F((dy + h) / h)
    zoff = zpx * zpx + zpy * zpy
    a = F((-2.0 * float(zpx)) / h)
    b = F((-2.0 * float(zpy)) / h)
    return a, b, zoff


def _depth(hw, plane, px, py):
    a, b, zoff = plane
    zx, zy = px + hw, py + hw
    return (a * zx + b * zy) + zoff


def _span(lo, hi, left, ps, n):
    i0 = math.ceil((float(lo) - left) / ps - 0.5)
    i1 = math.ceil((float(hi) - left) / ps - 0.5) - 1
    return max(i0, 0), min(i1, n - 1)


def compat_restated(scale, cell, sr, qr_d, pmin, mult, ox, oy, nrows, ncols, pts):
    qs = float(cell)
    ps = qs / scale
    qr = float(F(qr_d))                                  # the reference keeps the radius as float
    po = math.ceil((qr - math.floor(scale / 2.0) * ps) / ps) + 1
    xp, yp = ncols * scale + 2 * po, nrows * scale + 2 * po
    left = 0 - (qs / 2.0) - (po * ps)
    hw = F(((nrows - 1) * qs) / 2.0)
    zoffset = -1 * pmin
    rs = float(F(sr)) / math.sqrt(2.0)
    dep = np.full((yp, xp), np.inf, np.float32)
    col = np.zeros((yp, xp), np.uint32)
    cx = [F(left + (p + 0.5) * ps) for p in range(xp)]
    cy = [F(left + (p + 0.5) * ps) for p in range(yp)]
    for x, y, z in pts:                                   # draw order: later equal depths win
        dx, dy = x - float(F(ox)), y - float(F(oy))
        sx, sy = F(dx), F(dy)
        plane = _plane(hw, dx, dy)
        zc = np.uint32(int(math.floor(((z + zoffset) + 1) * mult)))
        i0, i1 = _span(F(float(sx) - rs), F(float(sx) + rs), left, ps, xp)
        j0, j1 = _span(F(float(sy) - rs), F(float(sy) + rs), left, ps, yp)
        for pj in range(j0, j1 + 1):
            for pi in range(i0, i1 + 1):
                d = _depth(hw, plane, cx[pi], cy[pj])
                if d <= dep[pj, pi]:
                    dep[pj, pi] = d
                    col[pj, pi] = zc
    rq = qr / math.sqrt(2.0)
    h = np.empty((nrows, ncols), np.float32)
    res = np.empty((nrows, ncols), np.int32)
    for j in range(nrows):
        for i in range(ncols):
            qx, qy = F(i * qs), F(j * qs)
            qplane = _plane(hw, i * qs, j * qs)
            i0, i1 = _span(F(float(qx) - rq), F(float(qx) + rq), left, ps, xp)
            j0, j1 = _span(F(float(qy) - rq), F(float(qy) + rq), left, ps, yp)
            numer, denom = 0, 0
            for pj in range(j0, j1 + 1):
                for pi in range(i0, i1 + 1):
                    if col[pj, pi] == 0:
                        continue
                    if _depth(hw, qplane, cx[pi], cy[pj]) <= dep[pj, pi]:
                        numer = (numer + int(col[pj, pi])) & 0xFFFFFFFF       # int32 sum with wrap
                        denom += 1
            if denom == 0:
                r = -9999 * mult
            else:
                sn = numer - (1 << 32) if numer >= 1 << 31 else numer
                r = (abs(sn) // denom) * (1 if sn >= 0 else -1)            # C truncation
            res[j, i] = r
            zz = 1.0 * r / mult
            if zz != -9999:
                zz = zz - zoffset - 1
            h[j, i] = F(zz)
    return h, res


@pytest.mark.parametrize("scale,cell,sr,qr,pmin,ncols,nrows,origin", [
    (5, 2.0, 5.0, 4.99, 0, 9, 7, (0.0, 0.0)),
    (2, 1.5, 4.0, 3.0, -7, 10, 8, (1000.0, 2000.0)),
    (1, 1.0, 2.5, 2.2, 3, 12, 9, (500100.0, 4100200.0)),
])
def test_compat_oracle_matches_an_independent_restatement(oracle, scale, cell, sr, qr, pmin, ncols, nrows, origin):
    rng = np.random.default_rng(scale * 100 + ncols)
    n = 60
    pts = np.stack([origin[0] + rng.uniform(-2, ncols * cell + 2, n), origin[1] + rng.uniform(-2, nrows * cell + 2, n),
                    rng.uniform(10, 40, n)], 1)
    pts = np.concatenate([pts, pts[:10]])                 # repeated positions: the later draw wins
    pts[-10:, 2] += 5.0
    mult = oracle.compat_multiplier(sr, scale, cell, float(pts[:, 2].max()), pmin)
    s = oracle.CompatSettings(scale=scale, cell_size=cell, site_radius=sr, query_radius=qr, point_min=pmin,
                              multiplier=mult, total_ncols=ncols, total_nrows=nrows)
    wp = oracle.CompatWP(origin_x=origin[0], origin_y=origin[1], grid_origin_x=0.0, grid_origin_y=0.0,
                         nrows=nrows, ncols=ncols)
    h, res = oracle.compat(s, wp, pts)
    h2, res2 = compat_restated(scale, cell, sr, qr, pmin, mult, origin[0], origin[1], nrows, ncols, pts)
    assert np.array_equal(res, res2)
    assert np.array_equal(h.view(np.uint32), h2.view(np.uint32))
    assert (res != -9999 * mult).mean() > 0.5
