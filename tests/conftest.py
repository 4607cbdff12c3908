"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

NATIVE = os.path.join(ROOT, "tests", "native")
EMU_SO = os.path.join(NATIVE, "libdnni_emu.so")


@pytest.fixture(scope="session", autouse=True)
def native_built():
    """Compile the in-tree native libraries if any source is newer."""
    from terranni_b200 import build
    build.build()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the engine through its C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


def _emu_deps():
    deps = [os.path.join(NATIVE, "dnni_emu.cu")]
    csrc = os.path.join(ROOT, "terranni_b200", "csrc")
    deps += [os.path.join(csrc, f) for f in ("dnni_search.cuh", "dnni_kernels.cuh", "dnni_plan.h")]
    deps.append(os.path.join(ROOT, "include", "dnni.h"))
    return deps


@pytest.fixture(scope="session")
def emu():
    """Host build of the engine's pipeline (same search/packing code)."""
    stale = not os.path.exists(EMU_SO) or any(os.path.getmtime(d) > os.path.getmtime(EMU_SO) for d in _emu_deps())
    if stale:
        cmd = ["/usr/local/cuda/bin/nvcc", "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
               "-gencode", "arch=compute_100a,code=sm_100a", "-o", EMU_SO, os.path.join(NATIVE, "dnni_emu.cu")]
        subprocess.run(cmd, check=True, capture_output=True)
    L = ctypes.CDLL(EMU_SO)
    L.emu_interpolate.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p]
    L.emu_interpolate.restype = ctypes.c_int

    def run(wp, xyz, gid=None, small_radius=0, bin_target=0):
        from oracle.oracle import raster_box
        xyz = np.ascontiguousarray(xyz, np.int32).reshape(-1, 3)
        if gid is not None:
            gid = np.ascontiguousarray(gid, np.uint32)
        x0, y0, x1, y1 = raster_box(wp)
        h = np.empty((wp.nrows, wp.ncols), np.float32)
        site = np.empty((y1 - y0, x1 - x0), np.uint32)
        r2 = np.empty((y1 - y0, x1 - x0), np.int32)
        info = np.zeros(8, np.int64)
        p = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
        rc = L.emu_interpolate(ctypes.addressof(wp), p(xyz), p(gid), xyz.shape[0], small_radius, bin_target,
                               p(h), p(site), p(r2), p(info))
        return rc, {"h": h, "site": site, "r2": r2,
                    "info": dict(zip(["packed", "K", "zbase", "bin_size", "big_pixels", "spans", "nodata",
                                      "max_r2"], info.tolist()))}
    return run


def load_golden():
    d = np.load(os.path.join(ROOT, "tests", "golden", "golden_cases.npz"))
    out = []
    for k, name in enumerate(d["names"]):
        p = f"c{k}_"
        wp = d[p + "wp"]
        zs = d[p + "zs"]
        out.append({
            "name": str(name), "xyz": d[p + "xyz"],
            "gid": d[p + "gid"] if bool(d[p + "has_gid"][0]) else None,
            "ncols": int(wp[0]), "nrows": int(wp[1]), "cell": int(wp[2]), "origin": (int(wp[3]), int(wp[4])),
            "raster": tuple(int(v) for v in wp[5:9]),
            "z_scale": float(zs[0]), "z_offset": float(zs[1]), "nodata": float(zs[2]),
            "site": d[p + "site"], "h": d[p + "h"], "Z": d[p + "Z"], "C": d[p + "C"],
        })
    return out


def golden_wp(mod, c):
    raster = c["raster"] if c["raster"] != (0, 0, 0, 0) else None
    return mod.make_wp(c["ncols"], c["nrows"], c["cell"], c["origin"][0], c["origin"][1], raster=raster,
                       z_scale=c["z_scale"], z_offset=c["z_offset"], nodata=c["nodata"])


def terrain_case(seed, side, n, cell=100, lakes=2, lake_r=(5.0, 20.0), nclusters=4, halo=None):
    """Small seeded terrain tile (LAS units, origin 0) for parity tests."""
    from terranni_b200 import synth
    ext = side * cell * synth.XY_SCALE
    xyz, lk = synth.generate(seed, n, ext, ext, kind="terrain", nclusters=nclusters, frac_uniform=0.7,
                             cluster_sigma=max(ext / 40, 0.5), nlakes=lakes, lake_rmin=lake_r[0] * cell / 100,
                             lake_rmax=lake_r[1] * cell / 100, relief=300.0, z_noise=0.1)
    return xyz
