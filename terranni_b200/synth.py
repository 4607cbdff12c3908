"""Seeded synthetic workloads (binding of csrc/synth.c).

The workloads are the five benchmark configurations of this engine: seeded
stand-ins with the stated shapes, sizes and value distributions; no public
dataset is involved.  All coordinates are int32 LAS units at 0.01 m.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdnni_synth.so")
BASE_SEED = 20261203
XY_SCALE = 0.01
Z_SCALE = 0.01


class SynthParams(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64), ("n", ctypes.c_int64),
        ("width", ctypes.c_double), ("height", ctypes.c_double),
        ("xy_scale", ctypes.c_double), ("z_scale", ctypes.c_double),
        ("kind", ctypes.c_int32), ("nclusters", ctypes.c_int32),
        ("frac_uniform", ctypes.c_double), ("cluster_sigma", ctypes.c_double),
        ("nlakes", ctypes.c_int32), ("octaves", ctypes.c_int32),
        ("lake_rmin", ctypes.c_double), ("lake_rmax", ctypes.c_double),
        ("relief", ctypes.c_double), ("z_noise", ctypes.c_double),
        ("hurst", ctypes.c_double), ("base_wavelength", ctypes.c_double),
        ("nthreads", ctypes.c_int32), ("pad", ctypes.c_int32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing (run python -m terranni_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        L.synth_generate.argtypes = [ctypes.POINTER(SynthParams), ctypes.c_void_p, ctypes.c_void_p]
        L.synth_generate.restype = ctypes.c_int
        _lib = L
    return _lib


def generate(seed, n, width, height, kind="terrain", nclusters=64, frac_uniform=0.7, cluster_sigma=20.0,
             nlakes=16, lake_rmin=50.0, lake_rmax=400.0, relief=300.0, z_noise=0.1, hurst=0.8, octaves=8,
             base_wavelength=None, nthreads=0, out=None):
    """-> (xyz int32 (n,3), lakes float64 (nlakes,3) as cx, cy, r in metres).
    out: optional C-contiguous int32 (n,3) array to generate into."""
    p = SynthParams()
    p.seed, p.n, p.width, p.height = int(seed), int(n), float(width), float(height)
    p.xy_scale, p.z_scale = XY_SCALE, Z_SCALE
    p.kind = 1 if kind == "sinusoid" else 0
    p.nclusters, p.frac_uniform, p.cluster_sigma = int(nclusters), float(frac_uniform), float(cluster_sigma)
    p.nlakes, p.octaves = int(nlakes), int(octaves)
    p.lake_rmin, p.lake_rmax = float(lake_rmin), float(lake_rmax)
    p.relief, p.z_noise, p.hurst = float(relief), float(z_noise), float(hurst)
    p.base_wavelength = float(base_wavelength if base_wavelength else max(width, height) / 2.0)
    p.nthreads = int(nthreads)
    if out is not None:
        if out.dtype != np.int32 or out.shape != (int(n), 3) or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a C-contiguous int32 (n, 3) array")
        xyz = out
    else:
        xyz = np.empty((int(n), 3), np.int32)
    lakes = np.zeros((max(int(nlakes), 1), 3), np.float64)
    rc = lib().synth_generate(ctypes.byref(p), xyz.ctypes.data_as(ctypes.c_void_p),
                              lakes.ctypes.data_as(ctypes.c_void_p))
    if rc:
        raise ValueError("synth_generate: bad parameters")
    return xyz, lakes[: int(nlakes)] if p.kind == 0 else lakes[:0]


def config1(seed=BASE_SEED):
    """512 x 512 grid at 1 m, 200k points, z = 4 sinusoids + N(0, 0.05 m)."""
    xyz, _ = generate(seed, 200_000, 512.0, 512.0, kind="sinusoid", z_noise=0.05)
    return {"xyz": xyz, "ncols": 512, "nrows": 512, "cell": 100,
            "las_offset": (500000.0, 4000000.0, 0.0)}


def config2(seed=BASE_SEED + 2, n=20_000_000, side=4096):
    """4096 x 4096 at 1 m, 20M points, 70% uniform + 30% in 64 clusters
    (sigma 20 m), 16 lakes of radius 50-400 m, fBm z (H 0.8, 8 octaves, 0-300 m)
    + N(0, 0.1 m)."""
    xyz, lakes = generate(seed, n, float(side), float(side), kind="terrain", nclusters=64, frac_uniform=0.7,
                          cluster_sigma=20.0, nlakes=16, lake_rmin=50.0, lake_rmax=400.0, relief=300.0,
                          z_noise=0.1)
    return {"xyz": xyz, "ncols": side, "nrows": side, "cell": 100, "lakes": lakes}


def config3(seed=BASE_SEED + 3, n=1_500_000_000, side=32768, out=None, nthreads=0):
    """Segment-streamed grid: side x side cells at 1 m, n points of the config-2
    generator scaled to the area (64 clusters and 16 lakes per 4096 m square,
    i.e. 4096 clusters and 1024 lakes at 32768 m)."""
    scale = (side / 4096.0) ** 2
    xyz, lakes = generate(seed, n, float(side), float(side), kind="terrain", nclusters=max(1, int(64 * scale)),
                          frac_uniform=0.7, cluster_sigma=20.0, nlakes=max(1, int(16 * scale)), lake_rmin=50.0,
                          lake_rmax=400.0, relief=300.0, z_noise=0.1, nthreads=nthreads, out=out)
    return {"xyz": xyz, "ncols": side, "nrows": side, "cell": 100, "lakes": lakes}


def config5(seed=BASE_SEED + 5, n=2_000_000_000, side_m=64000.0, out=None, nthreads=0):
    """Served cloud: n points over side_m x side_m metres (0.49 points/m^2 at
    the defaults), the config-2 generator scaled to the area (64 clusters and
    16 lakes per 4096 m square)."""
    scale = (side_m / 4096.0) ** 2
    xyz, lakes = generate(seed, n, side_m, side_m, kind="terrain", nclusters=max(1, int(64 * scale)),
                          frac_uniform=0.7, cluster_sigma=20.0, nlakes=max(1, int(16 * scale)), lake_rmin=50.0,
                          lake_rmax=400.0, relief=300.0, z_noise=0.1, base_wavelength=4096.0, nthreads=nthreads,
                          out=out)
    return {"xyz": xyz, "side_m": side_m, "lakes": lakes}


def served_requests(count, seed=BASE_SEED + 6, side_m=64000.0):
    """Request boxes: side log-uniform in 128 m - 8 km, cell 0.5/1/2 m, placed
    uniformly inside the cloud's area (LAS units at 0.01 m)."""
    rng = np.random.default_rng(seed)
    side = np.exp(rng.uniform(math.log(128.0), math.log(8192.0), count))
    cell = rng.choice(np.array([50, 100, 200]), count)
    out = []
    for k in range(count):
        n = max(1, int(round(side[k] * 100 / cell[k])))
        span = n * int(cell[k])
        x0 = int(rng.integers(0, max(1, int(side_m * 100) - span)))
        y0 = int(rng.integers(0, max(1, int(side_m * 100) - span)))
        out.append({"x0": x0, "y0": y0, "ncols": n, "nrows": n, "cell_size": int(cell[k])})
    return out


def mixed_tiles(count=4096, seed=BASE_SEED + 4, max_points=1_000_000):
    """Tile specs of the mixed batch: side log-uniform in [64, 1024] cells,
    cell 0.5/1/2 m, density log-uniform in [0.05, 8] points/cell,
    N = clamp(density * side^2, 1e3, 1e6), 0-4 lakes (radius 5-30 % of side)."""
    rng = np.random.default_rng(seed)
    side = np.exp(rng.uniform(math.log(64), math.log(1024), count)).astype(np.int64)
    cell = rng.choice(np.array([50, 100, 200]), count)
    dens = np.exp(rng.uniform(math.log(0.05), math.log(8.0), count))
    n = np.clip((dens * side * side).astype(np.int64), 1000, max_points)
    lakes = rng.integers(0, 5, count)
    seeds = rng.integers(1, 2 ** 62, count)
    return [{"side": int(side[i]), "cell": int(cell[i]), "n": int(n[i]), "lakes": int(lakes[i]),
             "seed": int(seeds[i])} for i in range(count)]


def tile_points(spec, out=None):
    ext = spec["side"] * spec["cell"] * XY_SCALE
    xyz, _ = generate(spec["seed"], spec["n"], ext, ext, kind="terrain", nclusters=8, frac_uniform=0.7,
                      cluster_sigma=max(ext / 50.0, 1.0), nlakes=spec["lakes"], lake_rmin=0.05 * ext,
                      lake_rmax=0.3 * ext, relief=300.0, z_noise=0.1, nthreads=1, out=out)
    return xyz


def tile_origin(k):
    """Absolute LAS origin of tile k of a mixed batch: tiles sit on a 64-wide
    lattice of 1.1 km pitch, so every tile has its own origin."""
    return (k % 64) * 110_000, (k // 64) * 110_000


def mixed_layout(specs):
    """Row offsets and output offsets of a mixed batch, in spec order."""
    pt = out = 0
    lay = []
    for k, s in enumerate(specs):
        ox, oy = tile_origin(k)
        lay.append({"pt": pt, "n": s["n"], "out": out, "side": s["side"], "cell": s["cell"], "origin": (ox, oy)})
        pt += s["n"]
        out += s["side"] * s["side"]
    return lay, pt, out


def fill_mixed(specs, lay, xyz, nthreads=None):
    """Generates every tile's points into its rows of xyz (absolute LAS
    coordinates) on a thread pool; returns each tile's point extent
    (x0, y0, x1, y1), absolute and inclusive."""
    from concurrent.futures import ThreadPoolExecutor
    nthreads = nthreads or os.cpu_count() or 1

    def one(k):
        s, L = specs[k], lay[k]
        rows = xyz[L["pt"]:L["pt"] + L["n"]]
        tile_points(s, out=rows)
        rows[:, 0] += L["origin"][0]
        rows[:, 1] += L["origin"][1]
        return (int(rows[:, 0].min()), int(rows[:, 1].min()), int(rows[:, 0].max()), int(rows[:, 1].max()))

    with ThreadPoolExecutor(nthreads) as ex:
        return list(ex.map(one, range(len(specs))))
