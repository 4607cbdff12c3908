"""ctypes binding of the CPU oracle (oracle/dnni_oracle.c).

TEST INFRASTRUCTURE ONLY.  Only the test suite, ``__graft_entry__.smoke()`` and
the cpu_baseline leg of ``bench.py`` import this module, and only as the
checker; the product library never calls it.  Parity is unpinned by the
reference's own tests (the reference ships none): the oracle is pinned by the
analytic known answers and brute-force restatements in ``tests/``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

NO_SITE = 0xFFFFFFFF


class WorkPackage(ctypes.Structure):
    """Same layout as ``dnni_workpackage`` (include/dnni.h)."""

    _fields_ = [
        ("ncols", ctypes.c_int32), ("nrows", ctypes.c_int32),
        ("cell_size", ctypes.c_int32),
        ("origin_x", ctypes.c_int32), ("origin_y", ctypes.c_int32),
        ("raster_x0", ctypes.c_int32), ("raster_y0", ctypes.c_int32),
        ("raster_x1", ctypes.c_int32), ("raster_y1", ctypes.c_int32),
        ("pad0", ctypes.c_int32),
        ("z_scale", ctypes.c_double), ("z_offset", ctypes.c_double),
        ("nodata", ctypes.c_float), ("pad1", ctypes.c_int32),
    ]


class CompatSettings(ctypes.Structure):
    _fields_ = [
        ("scale", ctypes.c_int32), ("cell_size", ctypes.c_float),
        ("site_radius", ctypes.c_float), ("query_radius", ctypes.c_double),
        ("point_min", ctypes.c_int32), ("multiplier", ctypes.c_int32),
        ("total_ncols", ctypes.c_int32), ("total_nrows", ctypes.c_int32),
    ]


class CompatWP(ctypes.Structure):
    _fields_ = [
        ("origin_x", ctypes.c_float), ("origin_y", ctypes.c_float),
        ("grid_origin_x", ctypes.c_float), ("grid_origin_y", ctypes.c_float),
        ("nrows", ctypes.c_int32), ("ncols", ctypes.c_int32),
    ]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "dnni_oracle.c"))
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i64 = ctypes.c_int64
        for name in ("orc_nearest", "orc_nearest_brute"):
            f = getattr(L, name)
            f.argtypes = [ctypes.POINTER(WorkPackage), P, P, i64, P, P, P]
            f.restype = ctypes.c_int
        for name in ("orc_interpolate", "orc_interpolate_brute"):
            f = getattr(L, name)
            f.argtypes = [ctypes.POINTER(WorkPackage), P, P, i64, P, P, P, P]
            f.restype = ctypes.c_int
        L.orc_work_stats.argtypes = [ctypes.POINTER(WorkPackage), P, P]
        L.orc_work_stats.restype = ctypes.c_int
        L.orc_gl_disagreement.argtypes = [ctypes.POINTER(WorkPackage), P, P, i64, ctypes.c_double,
                                          ctypes.c_int, i64, P]
        L.orc_gl_disagreement.restype = ctypes.c_int
        L.orc_compat.argtypes = [ctypes.POINTER(CompatSettings), ctypes.POINTER(CompatWP), P, i64, P, P]
        L.orc_compat.restype = ctypes.c_int
        L.orc_compat_multiplier.argtypes = [ctypes.c_float, ctypes.c_int32, ctypes.c_float,
                                            ctypes.c_double, ctypes.c_int32]
        L.orc_compat_multiplier.restype = ctypes.c_int32
        L.orc_interpolate_st.argtypes = [ctypes.POINTER(WorkPackage), P, P, i64, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.c_int32, ctypes.c_int, P, P, P]
        L.orc_interpolate_st.restype = ctypes.c_int
        L.orc_height.argtypes = [i64, i64, ctypes.c_double, ctypes.c_double, ctypes.c_float]
        L.orc_height.restype = ctypes.c_float
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def make_wp(ncols, nrows, cell_size, origin_x=0, origin_y=0, raster=None,
            z_scale=0.01, z_offset=0.0, nodata=-9999.0) -> WorkPackage:
    wp = WorkPackage()
    wp.ncols, wp.nrows, wp.cell_size = ncols, nrows, cell_size
    wp.origin_x, wp.origin_y = origin_x, origin_y
    if raster is not None:
        wp.raster_x0, wp.raster_y0, wp.raster_x1, wp.raster_y1 = raster
    wp.z_scale, wp.z_offset, wp.nodata = z_scale, z_offset, nodata
    return wp


def raster_box(wp: WorkPackage):
    if (wp.raster_x0, wp.raster_y0, wp.raster_x1, wp.raster_y1) == (0, 0, 0, 0):
        return 0, 0, wp.ncols, wp.nrows
    return wp.raster_x0, wp.raster_y0, wp.raster_x1, wp.raster_y1


def _prep(xyz, gid):
    xyz = np.ascontiguousarray(xyz, dtype=np.int32).reshape(-1, 3)
    if gid is not None:
        gid = np.ascontiguousarray(gid, dtype=np.uint32)
        assert gid.shape[0] == xyz.shape[0]
    return xyz, gid


def nearest(wp, xyz, gid=None, brute=False):
    """Exact nearest site per raster pixel -> (site_gid, site_z, r2) arrays
    shaped (raster rows, raster cols)."""
    xyz, gid = _prep(xyz, gid)
    x0, y0, x1, y1 = raster_box(wp)
    shape = (y1 - y0, x1 - x0)
    sg = np.empty(shape, np.uint32)
    sz = np.empty(shape, np.int32)
    r2 = np.empty(shape, np.int32)
    f = lib().orc_nearest_brute if brute else lib().orc_nearest
    rc = f(ctypes.byref(wp), _ptr(xyz), _ptr(gid), xyz.shape[0], _ptr(sg), _ptr(sz), _ptr(r2))
    if rc:
        raise ValueError(f"oracle nearest failed: {rc}")
    return sg, sz, r2


def interpolate(wp, xyz, gid=None, brute=False):
    """Canonical discrete NNI -> dict(h, site, Z, C)."""
    xyz, gid = _prep(xyz, gid)
    x0, y0, x1, y1 = raster_box(wp)
    h = np.empty((wp.nrows, wp.ncols), np.float32)
    site = np.empty((y1 - y0, x1 - x0), np.uint32)
    Z = np.empty((wp.nrows, wp.ncols), np.int64)
    C = np.empty((wp.nrows, wp.ncols), np.int64)
    f = lib().orc_interpolate_brute if brute else lib().orc_interpolate
    rc = f(ctypes.byref(wp), _ptr(xyz), _ptr(gid), xyz.shape[0], _ptr(h), _ptr(site), _ptr(Z), _ptr(C))
    if rc:
        raise ValueError(f"oracle interpolate failed: {rc}")
    return {"h": h, "site": site, "Z": Z, "C": C}


def interpolate_spacetime(wp, xyz, t, cur_time, time_radius, time_scale, brute=False):
    """Space-time canonical NNI (slices cur - rt .. cur + rt, lifted time
    distance, time_scale LAS units per time step) -> dict(h, Z, C)."""
    xyz = np.ascontiguousarray(xyz, np.int32).reshape(-1, 3)
    t = np.ascontiguousarray(t, np.int32).reshape(-1)
    if t.shape[0] != xyz.shape[0]:
        raise ValueError("one time per point")
    h = np.empty((wp.nrows, wp.ncols), np.float32)
    Z = np.empty((wp.nrows, wp.ncols), np.int64)
    C = np.empty((wp.nrows, wp.ncols), np.int64)
    rc = lib().orc_interpolate_st(ctypes.byref(wp), _ptr(xyz), _ptr(t), xyz.shape[0], int(cur_time),
                                  int(time_radius), int(time_scale), 1 if brute else 0, _ptr(h), _ptr(Z), _ptr(C))
    if rc:
        raise ValueError(f"oracle interpolate_spacetime failed: {rc}")
    return {"h": h, "Z": Z, "C": C}


def work_stats(wp, r2):
    out = np.zeros(3, np.int64)
    r2 = np.ascontiguousarray(r2, np.int32)
    lib().orc_work_stats(ctypes.byref(wp), _ptr(r2), _ptr(out))
    return {"spans": int(out[0]), "max_r2": int(out[1]), "pixels_with_site": int(out[2])}


def height(Z, C, z_scale, z_offset, nodata=-9999.0):
    return lib().orc_height(int(Z), int(C), z_scale, z_offset, nodata)


def exact_height_f64(Z, C, z_scale, z_offset):
    """FP64-or-better truth for the error figures: exact rational mean, one
    rounding to float64 at the end (numpy longdouble where available)."""
    Z = np.asarray(Z)
    C = np.asarray(C)
    with np.errstate(invalid="ignore", divide="ignore"):
        q = Z.astype(np.longdouble) / C.astype(np.longdouble)
        return (q * np.longdouble(z_scale) + np.longdouble(z_offset)).astype(np.float64)


def gl_disagreement(wp, xyz, gid=None, xy_scale=0.01, depth_bits=24, slack_units2=None):
    """Fraction of raster pixels whose site under the reference's float32
    lifted-plane depth test (emulated) differs from the exact nearest site."""
    xyz, gid = _prep(xyz, gid)
    if slack_units2 is None:
        hw_units = (wp.nrows - 1) * wp.cell_size / 2.0
        # float32 plane depth error ~ a few ulp of O(8) in normalised units;
        # 24-bit depth quantises 400/2^24 normalised units.  Generous slack:
        slack_units2 = int(max(2.0 ** -12 * hw_units * hw_units, 4 * wp.cell_size * wp.cell_size))
    out = np.zeros(3, np.int64)
    rc = lib().orc_gl_disagreement(ctypes.byref(wp), _ptr(xyz), _ptr(gid), xyz.shape[0], xy_scale,
                                   depth_bits, int(slack_units2), _ptr(out))
    if rc:
        raise ValueError(f"oracle gl_disagreement failed: {rc}")
    n = max(int(out[0]), 1)
    return {"pixels": int(out[0]), "site_differs": int(out[1]), "z_differs": int(out[2]),
            "site_frac": out[1] / n, "z_frac": out[2] / n}


def compat(settings: CompatSettings, cwp: CompatWP, pts_world):
    pts = np.ascontiguousarray(pts_world, dtype=np.float64).reshape(-1, 3)
    h = np.empty((cwp.nrows, cwp.ncols), np.float32)
    res = np.empty((cwp.nrows, cwp.ncols), np.int32)
    rc = lib().orc_compat(ctypes.byref(settings), ctypes.byref(cwp), _ptr(pts), pts.shape[0], _ptr(h), _ptr(res))
    if rc:
        raise ValueError(f"oracle compat failed: {rc}")
    return h, res


def compat_multiplier(site_radius, scale, cell_size, zmax, point_min):
    return lib().orc_compat_multiplier(site_radius, scale, cell_size, zmax, point_min)
