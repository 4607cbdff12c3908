"""Generates the golden known-answer fixtures in tests/golden/ (golden_cases.npz).

The reference ships no tests or fixtures, and it cannot be run here, so these
vectors come from a third, independent statement of the discrete
natural-neighbour rule: plain Python integers, brute force over every
(pixel, point) and (pixel, cell) pair, no shared code with the C oracle or the
CUDA engine.  Cases are small, analytic where possible (single site, bisector,
symmetric lattice, constant field, exact ties, empty input) and seeded random
otherwise.

Rule (reference: nni.cpp:171-230 site planes = nearest site per pixel;
nni.cpp:483-534 + cuda_nni.cu:407-503 query test |p-q|^2 <= |p-s(p)|^2 and
the numer/denom average):
  s(p)  = site minimising (d^2, gid, z);  R2 = floor(d^2 / cell^2)
  cell q gets z(s(p)) and 1 from every raster pixel p with |q-p|^2 <= R2(p)
  h     = float32(float64(Z) / float64(C) * z_scale + z_offset), nodata if C == 0

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import random

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_cases.npz")


def brute(case):
    ncols, nrows, cs = case["ncols"], case["nrows"], case["cell"]
    ox, oy = case["origin"]
    rx0, ry0, rx1, ry1 = case["raster"] if case["raster"] else (0, 0, ncols, nrows)
    pts = case["xyz"]
    gids = case["gid"] if case["gid"] is not None else list(range(len(pts)))
    ex = max(rx1, ncols) - min(rx0, 0)
    ey = max(ry1, nrows) - min(ry0, 0)
    cap = ex * ex + ey * ey
    site = []
    Z = [[0] * ncols for _ in range(nrows)]
    C = [[0] * ncols for _ in range(nrows)]
    for j in range(ry0, ry1):
        row = []
        for i in range(rx0, rx1):
            px, py = ox + i * cs, oy + j * cs
            best = None
            for k, (x, y, z) in enumerate(pts):
                d2 = (x - px) ** 2 + (y - py) ** 2
                key = (d2, gids[k], z)
                if best is None or key < best:
                    best = key
            if best is None:
                row.append(0xFFFFFFFF)
                continue
            row.append(best[1])
            R2 = min(best[0] // (cs * cs), cap)
            for qy in range(nrows):
                for qx in range(ncols):
                    if (qx - i) ** 2 + (qy - j) ** 2 <= R2:
                        Z[qy][qx] += best[2]
                        C[qy][qx] += 1
        site.append(row)
    h = np.empty((nrows, ncols), np.float32)
    for qy in range(nrows):
        for qx in range(ncols):
            if C[qy][qx] == 0:
                h[qy, qx] = np.float32(case["nodata"])
            else:
                v = float(Z[qy][qx]) / float(C[qy][qx])
                v = v * case["z_scale"]
                v = v + case["z_offset"]
                h[qy, qx] = np.float32(v)
    return (np.array(site, np.uint32).reshape(ry1 - ry0, rx1 - rx0), h,
            np.array(Z, np.int64), np.array(C, np.int64))


def cases():
    out = []

    def add(name, ncols, nrows, cell, xyz, origin=(0, 0), raster=None, gid=None, z_scale=0.01, z_offset=0.0,
            nodata=-9999.0):
        out.append(dict(name=name, ncols=ncols, nrows=nrows, cell=cell, xyz=[tuple(p) for p in xyz], origin=origin,
                        raster=raster, gid=gid, z_scale=z_scale, z_offset=z_offset, nodata=nodata))

    add("single_site", 9, 7, 100, [(430, 270, 1234)])
    add("two_site_bisector", 12, 5, 100, [(250, 200, 1000), (850, 200, 3000)])
    add("symmetric_lattice", 9, 9, 100, [(200 + 200 * a, 200 + 200 * b, 500 + 7 * a * b) for a in range(3) for b in range(3)])
    add("constant_field", 10, 8, 50, [(17 * k % 500, 31 * k % 400, 4242) for k in range(40)])
    add("exact_ties_duplicate_xy", 6, 6, 100, [(250, 250, 100), (250, 250, 900), (250, 250, 500)], gid=[7, 3, 5])
    add("equidistant_gid_tie", 7, 7, 100, [(300, 100, 10), (100, 300, 20), (500, 300, 30), (300, 500, 40)], gid=[4, 2, 9, 1])
    add("empty_input", 5, 4, 100, [])
    add("raster_halo", 6, 5, 100, [(50, 50, 600), (480, 420, -300), (260, 150, 42)], raster=(-3, -2, 9, 8))
    add("raster_offset_window", 8, 8, 100, [(150, 650, 11), (650, 150, 22), (900, 900, 33)], raster=(2, 2, 6, 6))
    add("far_outside_points", 6, 6, 100, [(-5000, -4000, 1), (9000, 300, 2), (300, 12000, 3)])
    add("utm_origin_cell1", 7, 6, 1, [(500003, 4000002, 77), (500001, 4000004, 88), (500006, 4000001, 99)],
        origin=(500000, 4000000))
    add("negative_coords_zoffset", 8, 6, 100, [(-150, -50, -2000), (420, 310, 1500), (700, -20, 300)],
        origin=(-200, -100), z_scale=0.001, z_offset=100.0, nodata=-1.0)
    rnd = random.Random(20261203)
    for t in range(12):
        nc, nr = rnd.randint(3, 14), rnd.randint(3, 14)
        cs = rnd.choice([1, 3, 50, 100])
        n = rnd.randint(1, 30)
        xyz = [(rnd.randint(-2 * cs, (nc + 2) * cs), rnd.randint(-2 * cs, (nr + 2) * cs), rnd.randint(-3000, 30000))
               for _ in range(n)]
        raster = None
        if t % 3 == 1:
            raster = (-rnd.randint(0, 3), -rnd.randint(0, 3), nc + rnd.randint(0, 3), nr + rnd.randint(0, 3))
        gid = None
        if t % 4 == 2:
            gid = rnd.sample(range(1000), n)
        add(f"random_{t}", nc, nr, cs, xyz, raster=raster, gid=gid)
    return out


def main():
    arrays = {}
    names = []
    for k, c in enumerate(cases()):
        site, h, Z, C = brute(c)
        p = f"c{k}_"
        names.append(c["name"])
        xyz = np.array(c["xyz"], np.int32).reshape(-1, 3)
        arrays[p + "xyz"] = xyz
        arrays[p + "gid"] = np.array(c["gid"] if c["gid"] is not None else [], np.uint32)
        arrays[p + "has_gid"] = np.array([c["gid"] is not None], np.bool_)
        arrays[p + "wp"] = np.array([c["ncols"], c["nrows"], c["cell"], c["origin"][0], c["origin"][1],
                                     *(c["raster"] if c["raster"] else (0, 0, 0, 0))], np.int64)
        arrays[p + "zs"] = np.array([c["z_scale"], c["z_offset"], c["nodata"]], np.float64)
        arrays[p + "site"] = site
        arrays[p + "h"] = h
        arrays[p + "Z"] = Z
        arrays[p + "C"] = C
    arrays["names"] = np.array(names)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {len(names)} cases to {OUT}")


if __name__ == "__main__":
    main()
