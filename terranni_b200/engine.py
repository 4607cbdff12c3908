"""Python binding of the engine's C ABI (include/dnni.h) via ctypes.

This is plumbing for the test suite, the smoke entry and ``bench.py``; the
drop-in boundary itself is the C ABI and the C++ ``nni::`` shim.  The native
library is required: if ``libdnni.so`` is missing every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdnni.so")

NO_SITE = 0xFFFFFFFF
F_TIMING = 1

STATUS = {
    0: "DNNI_OK", 1: "DNNI_E_INVAL", 2: "DNNI_E_NOMEM", 3: "DNNI_E_TIMEOUT", 4: "DNNI_E_CUDA",
    5: "DNNI_E_RANGE", 6: "DNNI_E_STATE", 7: "DNNI_E_IO", 8: "DNNI_E_CANCELLED", 9: "DNNI_E_BUSY",
    10: "DNNI_E_SCRATCH",
}


class DnniError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {message}")


class Settings(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("small_radius", ctypes.c_int32),
                ("bin_target", ctypes.c_int32), ("flags", ctypes.c_int32),
                ("mem_budget", ctypes.c_uint64)]


class WorkPackage(ctypes.Structure):
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


class Stats(ctypes.Structure):
    _fields_ = [
        ("ms_total", ctypes.c_double), ("ms_bin", ctypes.c_double), ("ms_nearest", ctypes.c_double),
        ("ms_scatter", ctypes.c_double), ("ms_finalize", ctypes.c_double),
        ("n_points", ctypes.c_int64), ("n_cells", ctypes.c_int64), ("n_pixels", ctypes.c_int64),
        ("big_pixels", ctypes.c_int64), ("spans", ctypes.c_int64), ("nodata_cells", ctypes.c_int64),
        ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
        ("max_r2", ctypes.c_int32), ("packed", ctypes.c_int32), ("bin_size", ctypes.c_int32),
        ("pad", ctypes.c_int32), ("evals_dense", ctypes.c_int64), ("evals_far", ctypes.c_int64),
        ("span_hist", ctypes.c_int64 * 16), ("ms_dense", ctypes.c_double), ("ms_far", ctypes.c_double),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("pad", "span_hist")}
        d["span_hist"] = list(self.span_hist)
        return d


class Tile(ctypes.Structure):
    _fields_ = [
        ("wp", WorkPackage),
        ("pt_offset", ctypes.c_int64), ("pt_count", ctypes.c_int64),
        ("ext_x0", ctypes.c_int32), ("ext_y0", ctypes.c_int32),
        ("ext_x1", ctypes.c_int32), ("ext_y1", ctypes.c_int32),
        ("out_offset", ctypes.c_int64), ("site_offset", ctypes.c_int64),
    ]


class BatchOptions(ctypes.Structure):
    _fields_ = [("small_radius", ctypes.c_int32), ("bin_target", ctypes.c_int32),
                ("use_graph", ctypes.c_int32), ("order_by_cost", ctypes.c_int32),
                ("span_window", ctypes.c_int32), ("far_group", ctypes.c_int32),
                ("dense_band", ctypes.c_int32)]


class Segment(ctypes.Structure):
    _fields_ = [("ncols", ctypes.c_int32), ("nrows", ctypes.c_int32), ("cell_size", ctypes.c_int32),
                ("origin_x", ctypes.c_int32), ("origin_y", ctypes.c_int32), ("tile", ctypes.c_int32),
                ("halo", ctypes.c_int32), ("tiles_per_batch", ctypes.c_int32),
                ("z_scale", ctypes.c_double), ("z_offset", ctypes.c_double),
                ("nodata", ctypes.c_float), ("small_radius", ctypes.c_int32),
                ("part", ctypes.c_int32), ("parts", ctypes.c_int32)]


class SegmentStats(ctypes.Structure):
    _fields_ = [("ms_total", ctypes.c_double), ("ms_upload", ctypes.c_double), ("ms_bucket", ctypes.c_double),
                ("ms_bound", ctypes.c_double), ("ms_tiles", ctypes.c_double), ("points", ctypes.c_int64), ("cells", ctypes.c_int64), ("tiles", ctypes.c_int64),
                ("tile_runs", ctypes.c_int64), ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
                ("max_halo", ctypes.c_int32), ("batches", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOptions(ctypes.Structure):
    _fields_ = [("bucket", ctypes.c_int32), ("fine", ctypes.c_int32), ("slots", ctypes.c_int32),
                ("max_batch", ctypes.c_int32), ("slot_bytes", ctypes.c_uint64), ("small_radius", ctypes.c_int32),
                ("bin_target", ctypes.c_int32)]


class Request(ctypes.Structure):
    _fields_ = [("x0", ctypes.c_int32), ("y0", ctypes.c_int32), ("ncols", ctypes.c_int32), ("nrows", ctypes.c_int32),
                ("cell_size", ctypes.c_int32), ("pad0", ctypes.c_int32), ("z_scale", ctypes.c_double),
                ("z_offset", ctypes.c_double), ("nodata", ctypes.c_float), ("pad1", ctypes.c_int32),
                ("out_h", ctypes.c_void_p), ("out_site", ctypes.c_void_p)]


class RequestResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("halo", ctypes.c_int32), ("ms_queue", ctypes.c_double),
                ("ms_latency", ctypes.c_double), ("points", ctypes.c_int64), ("cells", ctypes.c_int64),
                ("batch_size", ctypes.c_int32), ("runs", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("batches", ctypes.c_int64), ("cells", ctypes.c_int64), ("points", ctypes.c_int64),
                ("resident_bytes", ctypes.c_int64), ("ms_build", ctypes.c_double),
                ("ms_device_busy", ctypes.c_double), ("ms_device_overlap", ctypes.c_double),
                ("ms_device_span", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class LasHeader(ctypes.Structure):
    _fields_ = [("version_major", ctypes.c_uint8), ("version_minor", ctypes.c_uint8),
                ("point_format", ctypes.c_uint8), ("pad0", ctypes.c_uint8), ("record_length", ctypes.c_uint16),
                ("pad1", ctypes.c_uint16), ("offset_to_points", ctypes.c_uint32), ("n_points", ctypes.c_uint64),
                ("scale", ctypes.c_double * 3), ("offset", ctypes.c_double * 3), ("min", ctypes.c_double * 3),
                ("max", ctypes.c_double * 3)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("pad")}
        for k in ("scale", "offset", "min", "max"):
            d[k] = list(d[k])
        return d


class CompatSettings(ctypes.Structure):
    _fields_ = [("scale", ctypes.c_int32), ("cell_size", ctypes.c_float), ("site_radius", ctypes.c_float),
                ("pad0", ctypes.c_int32), ("query_radius", ctypes.c_double), ("point_min", ctypes.c_int32),
                ("multiplier", ctypes.c_int32), ("total_ncols", ctypes.c_int32), ("total_nrows", ctypes.c_int32)]


class StOptions(ctypes.Structure):
    """dnni_st_options: space-time interpolation settings."""
    _fields_ = [("cur_time", ctypes.c_int32), ("time_radius", ctypes.c_int32), ("time_scale", ctypes.c_int32),
                ("pad", ctypes.c_int32)]


class CompatWP(ctypes.Structure):
    _fields_ = [("origin_x", ctypes.c_float), ("origin_y", ctypes.c_float), ("grid_origin_x", ctypes.c_float),
                ("grid_origin_y", ctypes.c_float), ("nrows", ctypes.c_int32), ("ncols", ctypes.c_int32)]


class Peaks(ctypes.Structure):
    _fields_ = [("int_ops_per_s", ctypes.c_double), ("smem_atomics_per_s", ctypes.c_double),
                ("l2_red64_per_s", ctypes.c_double), ("sm_clock_mhz", ctypes.c_double),
                ("sm_count", ctypes.c_int32), ("pad", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class TuneTrial(ctypes.Structure):
    _fields_ = [("small_radius", ctypes.c_int32), ("bin_target", ctypes.c_int32), ("ms", ctypes.c_float),
                ("span_window", ctypes.c_int32), ("far_group", ctypes.c_int32), ("dense_band", ctypes.c_int32)]


class TuneReport(ctypes.Structure):
    _fields_ = [("ntrials", ctypes.c_int32), ("best", ctypes.c_int32), ("sample_tiles", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("ms_default", ctypes.c_double), ("trial", TuneTrial * 32)]

    def as_dict(self):
        t = [{"small_radius": self.trial[k].small_radius, "bin_target": self.trial[k].bin_target,
              "span_window": self.trial[k].span_window, "far_group": self.trial[k].far_group,
              "dense_band": self.trial[k].dense_band, "ms": self.trial[k].ms} for k in range(self.ntrials)]
        return {"sample_tiles": self.sample_tiles, "ms_default": self.ms_default,
                "best": t[self.best] if t else None, "trials": t}


# every symbol include/dnni.h declares, with (argtypes, restype)
_P = ctypes.c_void_p
_SIGS = {
    "dnni_version": ([], ctypes.c_int32),
    "dnni_init": ([ctypes.POINTER(Settings), ctypes.POINTER(_P)], ctypes.c_int),
    "dnni_destroy": ([_P], ctypes.c_int),
    "dnni_last_error": ([_P], ctypes.c_char_p),
    "dnni_setup_run": ([_P, ctypes.POINTER(WorkPackage), ctypes.c_int64], ctypes.c_int),
    "dnni_interpolate_segment": ([_P, ctypes.POINTER(WorkPackage), _P, _P, ctypes.c_int64, _P, _P,
                                  ctypes.POINTER(Stats)], ctypes.c_int),
    "dnni_interpolate_segment_device": ([_P, ctypes.POINTER(WorkPackage), _P, _P, ctypes.c_int64, _P, _P, _P,
                                         ctypes.POINTER(Stats)], ctypes.c_int),
    "dnni_interpolate_segment_device_noalloc": ([ctypes.POINTER(WorkPackage), _P, _P, ctypes.c_int64, _P, _P, _P],
                                                ctypes.c_int),
    "dnni_clear": ([_P], ctypes.c_int),
    "dnni_print_times": ([_P], ctypes.c_int),
    "dnni_host_alloc": ([ctypes.c_size_t, ctypes.POINTER(_P)], ctypes.c_int),
    "dnni_host_free": ([_P], ctypes.c_int),
    "dnni_measure_peaks": ([ctypes.c_int32, ctypes.POINTER(Peaks)], ctypes.c_int),
    "dnni_partition_contiguous": ([_P, ctypes.c_int32, ctypes.c_int32, _P], ctypes.c_int),
    "dnni_batch_create": ([_P, ctypes.POINTER(Tile), ctypes.c_int32, ctypes.POINTER(BatchOptions),
                           ctypes.POINTER(_P)], ctypes.c_int),
    "dnni_batch_run_device": ([_P, _P, _P, _P, _P, _P, ctypes.POINTER(Stats)], ctypes.c_int),
    "dnni_batch_run": ([_P, _P, _P, ctypes.c_int64, _P, _P, ctypes.POINTER(Stats)], ctypes.c_int),
    "dnni_batch_destroy": ([_P], ctypes.c_int),
    "dnni_segment_run": ([_P, ctypes.POINTER(Segment), _P, ctypes.c_int64, _P, _P, ctypes.POINTER(SegmentStats)],
                         ctypes.c_int),
    "dnni_server_create": ([_P, _P, ctypes.c_int64, ctypes.POINTER(ServerOptions), ctypes.POINTER(_P)], ctypes.c_int),
    "dnni_server_submit": ([_P, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    "dnni_server_wait": ([_P, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(RequestResult)], ctypes.c_int),
    "dnni_server_get_stats": ([_P, ctypes.POINTER(ServerStats)], ctypes.c_int),
    "dnni_server_destroy": ([_P], ctypes.c_int),
    "dnni_las_read_header": ([ctypes.c_char_p, ctypes.POINTER(LasHeader)], ctypes.c_int),
    "dnni_las_read": ([ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64, _P, _P, ctypes.c_int32], ctypes.c_int),
    "dnni_las_write": ([ctypes.c_char_p, _P, _P, ctypes.c_int64, _P, _P], ctypes.c_int),
    "dnni_write_asc": ([ctypes.c_char_p, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                        ctypes.c_double, ctypes.c_float, ctypes.c_int32], ctypes.c_int),
    "dnni_write_grid_bin": ([ctypes.c_char_p, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                             ctypes.c_double, ctypes.c_float], ctypes.c_int),
    "dnni_interpolate_spacetime": ([_P, ctypes.POINTER(WorkPackage), ctypes.POINTER(StOptions), _P, _P,
                                    ctypes.c_int64, _P, _P], ctypes.c_int),
    "dnni_interpolate_spacetime_device": ([_P, ctypes.POINTER(WorkPackage), ctypes.POINTER(StOptions), _P, _P,
                                           ctypes.c_int64, _P, _P, _P], ctypes.c_int),
    "dnni_interpolate_compat_device": ([_P, ctypes.POINTER(CompatSettings), ctypes.POINTER(CompatWP), _P,
                                        ctypes.c_int64, _P, _P, _P], ctypes.c_int),
    "dnni_interpolate_compat": ([_P, ctypes.POINTER(CompatSettings), ctypes.POINTER(CompatWP), _P, ctypes.c_int64,
                                 _P, _P], ctypes.c_int),
    "dnni_batch_autotune": ([_P, ctypes.POINTER(Tile), ctypes.c_int32, _P, _P, ctypes.c_int32,
                             ctypes.POINTER(BatchOptions), ctypes.POINTER(TuneReport)], ctypes.c_int),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"native engine not built: {LIB_PATH} is missing (run python -m terranni_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def partition_contiguous(costs, parts):
    """dnni_partition_contiguous -> first (parts + 1 ints): part p owns items
    [first[p], first[p+1]) of a cost-balanced contiguous split."""
    c = np.ascontiguousarray(costs, dtype=np.int64)
    first = np.zeros(int(parts) + 1, np.int32)
    _rc(lib().dnni_partition_contiguous(c.ctypes.data if c.size else None, c.size, int(parts),
                                        first.ctypes.data), "dnni_partition_contiguous")
    return first


def measure_peaks(device=0):
    """dnni_measure_peaks -> dict: measured integer multiply-add, shared-memory
    atomic and L2 64-bit reduction throughput of the device (lane ops/s)."""
    p = Peaks()
    _rc(lib().dnni_measure_peaks(int(device), ctypes.byref(p)), "dnni_measure_peaks")
    return p.as_dict()


def make_wp(ncols, nrows, cell_size, origin_x=0, origin_y=0, raster=None, z_scale=0.01, z_offset=0.0,
            nodata=-9999.0) -> WorkPackage:
    wp = WorkPackage()
    wp.ncols, wp.nrows, wp.cell_size = int(ncols), int(nrows), int(cell_size)
    wp.origin_x, wp.origin_y = int(origin_x), int(origin_y)
    if raster is not None:
        wp.raster_x0, wp.raster_y0, wp.raster_x1, wp.raster_y1 = (int(v) for v in raster)
    wp.z_scale, wp.z_offset, wp.nodata = float(z_scale), float(z_offset), float(nodata)
    return wp


def raster_box(wp: WorkPackage):
    if (wp.raster_x0, wp.raster_y0, wp.raster_x1, wp.raster_y1) == (0, 0, 0, 0):
        return 0, 0, wp.ncols, wp.nrows
    return wp.raster_x0, wp.raster_y0, wp.raster_x1, wp.raster_y1


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):          # torch tensor
        return a.data_ptr()
    return a.ctypes.data_as(ctypes.c_void_p).value


class Engine:
    """One dnni context (one device, one host thread at a time)."""

    def __init__(self, device=0, small_radius=0, bin_target=0, flags=0, mem_budget=0):
        s = Settings(device, small_radius, bin_target, flags, mem_budget)
        h = _P()
        rc = lib().dnni_init(ctypes.byref(s), ctypes.byref(h))
        if rc:
            raise DnniError(rc, "dnni_init failed")
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().dnni_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc:
            msg = lib().dnni_last_error(self._h)
            raise DnniError(rc, msg.decode() if msg else "")

    def setup_run(self, wp, max_points):
        self._check(lib().dnni_setup_run(self._h, ctypes.byref(wp), int(max_points)))

    def interpolate(self, wp: WorkPackage, xyz, gid=None, site=False, out_h=None):
        """Host-buffer call (dnni_interpolate_segment) -> (h, site_map, stats)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.int32).reshape(-1, 3)
        if gid is not None:
            gid = np.ascontiguousarray(gid, dtype=np.uint32)
        h = out_h if out_h is not None else np.empty((wp.nrows, wp.ncols), np.float32)
        x0, y0, x1, y1 = raster_box(wp)
        sm = np.empty((y1 - y0, x1 - x0), np.uint32) if site else None
        st = Stats()
        self._check(lib().dnni_interpolate_segment(self._h, ctypes.byref(wp), _ptr(xyz), _ptr(gid),
                                                   xyz.shape[0], _ptr(h), _ptr(sm), ctypes.byref(st)))
        return h, sm, st

    def interpolate_spacetime(self, wp: WorkPackage, xyz, t, cur_time, time_radius, time_scale, out_h=None):
        """dnni_interpolate_spacetime (timeRadius > 0) -> (h, stats)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.int32).reshape(-1, 3)
        t = np.ascontiguousarray(t, dtype=np.int32).reshape(-1)
        if t.shape[0] != xyz.shape[0]:
            raise ValueError("one time per point")
        h = out_h if out_h is not None else np.empty((wp.nrows, wp.ncols), np.float32)
        st = Stats()
        opt = StOptions(int(cur_time), int(time_radius), int(time_scale), 0)
        self._check(lib().dnni_interpolate_spacetime(self._h, ctypes.byref(wp), ctypes.byref(opt), _ptr(xyz), _ptr(t),
                                                     xyz.shape[0], _ptr(h), ctypes.byref(st)))
        return h, st

    def interpolate_spacetime_device(self, wp: WorkPackage, d_xyz, d_t, n, d_h, cur_time, time_radius, time_scale,
                                     stream=None, stats=True):
        """dnni_interpolate_spacetime_device: device buffers (torch tensors or
        raw addresses), queued on `stream` (raw cudaStream_t)."""
        st = Stats() if stats else None
        opt = StOptions(int(cur_time), int(time_radius), int(time_scale), 0)
        self._check(lib().dnni_interpolate_spacetime_device(
            self._h, ctypes.byref(wp), ctypes.byref(opt), _ptr(d_xyz), _ptr(d_t), int(n), _ptr(d_h), stream,
            ctypes.byref(st) if st is not None else None))
        return st

    def interpolate_device(self, wp: WorkPackage, d_xyz, n, d_h, d_gid=None, d_site=None, stream=None,
                           stats=True):
        """Device-buffer call (dnni_interpolate_segment_device).  Buffers are
        torch CUDA tensors or raw device addresses; stream is a raw
        cudaStream_t value (e.g. torch.cuda.current_stream().cuda_stream)."""
        st = Stats() if stats else None
        self._check(lib().dnni_interpolate_segment_device(
            self._h, ctypes.byref(wp), _ptr(d_xyz), _ptr(d_gid), int(n), _ptr(d_h), _ptr(d_site),
            stream, ctypes.byref(st) if st is not None else None))
        return st

    def batch(self, tiles, small_radius=0, bin_target=0, use_graph=False, order_by_cost=False, span_window=0,
              far_group=0, dense_band=0):
        """Plans a batch of tiles (dnni_batch_create) -> Batch."""
        return Batch(self, tiles, small_radius, bin_target, use_graph, order_by_cost, span_window, far_group,
                     dense_band)

    def autotune(self, tiles, d_xyz, d_gid=None, sample_tiles=256, small_radius=0, bin_target=0, span_window=0,
                 far_group=0, dense_band=0):
        """dnni_batch_autotune -> (dict of the chosen batch options, report dict)."""
        arr = (Tile * len(tiles))(*tiles)
        opt = BatchOptions(int(small_radius), int(bin_target), 0, 0, int(span_window), int(far_group),
                           int(dense_band))
        rep = TuneReport()
        self._check(lib().dnni_batch_autotune(self._h, arr, len(tiles), _ptr(d_xyz), _ptr(d_gid), int(sample_tiles),
                                              ctypes.byref(opt), ctypes.byref(rep)))
        return ({"small_radius": opt.small_radius, "bin_target": opt.bin_target, "span_window": opt.span_window,
                 "far_group": opt.far_group, "dense_band": opt.dense_band}, rep.as_dict())

    def segment_run(self, xyz, ncols, nrows, cell_size, origin=(0, 0), tile=0, halo=0, tiles_per_batch=0,
                    z_scale=0.01, z_offset=0.0, nodata=-9999.0, small_radius=0, site=False, out_h=None, part=0,
                    parts=0):
        """dnni_segment_run: the whole grid (or, with parts > 1, the tiles of
        part `part`) from host points in tiles with halos -> (h, site map or
        None, SegmentStats)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.int32).reshape(-1, 3)
        sg = Segment(int(ncols), int(nrows), int(cell_size), int(origin[0]), int(origin[1]), int(tile), int(halo),
                     int(tiles_per_batch), float(z_scale), float(z_offset), float(nodata), int(small_radius),
                     int(part), int(parts))
        h = out_h if out_h is not None else np.empty((nrows, ncols), np.float32)
        sm = np.empty((nrows, ncols), np.uint32) if site else None
        st = SegmentStats()
        self._check(lib().dnni_segment_run(self._h, ctypes.byref(sg), _ptr(xyz), xyz.shape[0], _ptr(h), _ptr(sm),
                                           ctypes.byref(st)))
        return h, sm, st

    def server(self, xyz, **options):
        """dnni_server_create over host points (absolute LAS xyz) -> Server."""
        return Server(self, xyz, **options)

    def interpolate_compat(self, settings: CompatSettings, wp: CompatWP, pts_world):
        """dnni_interpolate_compat (the reference's default semantics) ->
        (heights, int32 division results)."""
        pts = np.ascontiguousarray(pts_world, dtype=np.float64).reshape(-1, 3)
        h = np.empty((wp.nrows, wp.ncols), np.float32)
        res = np.empty((wp.nrows, wp.ncols), np.int32)
        self._check(lib().dnni_interpolate_compat(self._h, ctypes.byref(settings), ctypes.byref(wp), _ptr(pts),
                                                  pts.shape[0], _ptr(h), _ptr(res)))
        return h, res

    def interpolate_compat_device(self, settings: CompatSettings, wp: CompatWP, d_pts, n, d_h, d_res=None,
                                  stream=None):
        """dnni_interpolate_compat_device: device buffers, queued on `stream`."""
        self._check(lib().dnni_interpolate_compat_device(self._h, ctypes.byref(settings), ctypes.byref(wp),
                                                         _ptr(d_pts), int(n), _ptr(d_h), _ptr(d_res), stream))

    def clear(self):
        self._check(lib().dnni_clear(self._h))

    def print_times(self):
        self._check(lib().dnni_print_times(self._h))


def make_tile(wp: WorkPackage, pt_offset, pt_count, out_offset, site_offset=-1, extent=None) -> Tile:
    """One batch entry; extent = absolute (x0, y0, x1, y1) LAS box of its
    points, None = the raster."""
    t = Tile()
    t.wp = wp
    t.pt_offset, t.pt_count = int(pt_offset), int(pt_count)
    if extent is not None:
        t.ext_x0, t.ext_y0, t.ext_x1, t.ext_y1 = (int(v) for v in extent)
    t.out_offset, t.site_offset = int(out_offset), int(site_offset)
    return t


class Batch:
    """A planned batch of tiles (dnni_batch); runs many times."""

    def __init__(self, eng: Engine, tiles, small_radius=0, bin_target=0, use_graph=False, order_by_cost=False,
                 span_window=0, far_group=0, dense_band=0):
        self._eng = eng
        arr = (Tile * len(tiles))(*tiles)
        opt = BatchOptions(int(small_radius), int(bin_target), int(bool(use_graph)), int(bool(order_by_cost)),
                           int(span_window), int(far_group), int(dense_band))
        h = _P()
        eng._check(lib().dnni_batch_create(eng.handle, arr, len(tiles), ctypes.byref(opt), ctypes.byref(h)))
        self._h = h
        self.tiles = list(tiles)

    def close(self):
        if self._h:
            lib().dnni_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run_device(self, d_xyz, d_h, d_gid=None, d_site=None, stream=None, stats=False):
        """dnni_batch_run_device: queued on `stream` (a raw cudaStream_t, e.g.
        torch.cuda.current_stream().cuda_stream; None = the context's own
        stream) and returns before the kernels finish unless stats is asked
        for (which synchronises)."""
        st = Stats() if stats else None
        self._eng._check(lib().dnni_batch_run_device(self._h, _ptr(d_xyz), _ptr(d_gid), _ptr(d_h), _ptr(d_site),
                                                     stream, ctypes.byref(st) if st is not None else None))
        return st

    def run(self, xyz, out_h, gid=None, out_site=None, stats=True):
        xyz = np.ascontiguousarray(xyz, dtype=np.int32).reshape(-1, 3)
        if gid is not None:
            gid = np.ascontiguousarray(gid, dtype=np.uint32)
        st = Stats() if stats else None
        self._eng._check(lib().dnni_batch_run(self._h, _ptr(xyz), _ptr(gid), xyz.shape[0], _ptr(out_h),
                                              _ptr(out_site), ctypes.byref(st) if st is not None else None))
        return st


class Server:
    """DEM requests against a resident cloud (dnni_server_*)."""

    def __init__(self, eng: Engine, xyz, bucket=0, fine=0, slots=0, max_batch=0, slot_bytes=0, small_radius=0,
                 bin_target=0):
        import threading
        self._eng = eng
        xyz = np.ascontiguousarray(xyz, dtype=np.int32).reshape(-1, 3)
        o = ServerOptions(int(bucket), int(fine), int(slots), int(max_batch), int(slot_bytes), int(small_radius),
                          int(bin_target))
        h = _P()
        eng._check(lib().dnni_server_create(eng.handle, _ptr(xyz), xyz.shape[0], ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._bufs = {}
        self._mu = threading.Lock()

    def submit(self, x0, y0, ncols, nrows, cell_size, site=False, z_scale=0.01, z_offset=0.0, nodata=-9999.0,
               out_h=None, out_site=None):
        """Queues a request; returns its ticket.  Buffers (numpy, pinned or
        not) are kept alive until wait() returns them."""
        h = out_h if out_h is not None else np.empty((nrows, ncols), np.float32)
        sm = out_site if out_site is not None else (np.empty((nrows, ncols), np.uint32) if site else None)
        r = Request(int(x0), int(y0), int(ncols), int(nrows), int(cell_size), 0, float(z_scale), float(z_offset),
                    float(nodata), 0, _ptr(h), _ptr(sm))
        t = ctypes.c_uint64()
        rc = lib().dnni_server_submit(self._h, ctypes.byref(r), ctypes.byref(t))
        if rc:
            raise DnniError(rc, "dnni_server_submit")
        with self._mu:
            self._bufs[t.value] = (h, sm)
        return t.value

    def wait(self, ticket, timeout=-1.0):
        """-> (heights, site map or None, result dict); raises DnniError when
        the request failed (its result dict is on the exception)."""
        res = RequestResult()
        rc = lib().dnni_server_wait(self._h, int(ticket), float(timeout), ctypes.byref(res))
        if rc == 3:                      # DNNI_E_TIMEOUT: still pending
            raise DnniError(rc, "timeout")
        with self._mu:
            h, sm = self._bufs.pop(ticket)
        if rc:
            e = DnniError(rc, "request failed")
            e.result = res.as_dict()
            raise e
        return h, sm, res.as_dict()

    def stats(self):
        st = ServerStats()
        self._eng._check(lib().dnni_server_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def close(self):
        if self._h:
            lib().dnni_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---- host I/O (no device needed) ----

def _rc(rc, what):
    if rc:
        raise DnniError(rc, what)


def las_read_header(path):
    h = LasHeader()
    _rc(lib().dnni_las_read_header(os.fsencode(path), ctypes.byref(h)), f"dnni_las_read_header {path}")
    return h.as_dict()


def las_read(path, first=0, count=None, intensity=False, out=None, nthreads=0):
    """Raw record integers (n, 3) int32 of records [first, first+count); with
    intensity also the (n,) uint16 intensities."""
    hd = las_read_header(path)
    if count is None:
        count = hd["n_points"] - first
    xyz = out if out is not None else np.empty((count, 3), np.int32)
    it = np.empty(count, np.uint16) if intensity else None
    _rc(lib().dnni_las_read(os.fsencode(path), int(first), int(count), _ptr(xyz), _ptr(it), int(nthreads)),
        f"dnni_las_read {path}")
    return (xyz, it) if intensity else xyz


def las_write(path, xyz, intensity=None, scale=(0.01, 0.01, 0.01), offset=(0.0, 0.0, 0.0)):
    xyz = np.ascontiguousarray(xyz, np.int32).reshape(-1, 3)
    if intensity is not None:
        intensity = np.ascontiguousarray(intensity, np.uint16)
    sc = (ctypes.c_double * 3)(*scale)
    of = (ctypes.c_double * 3)(*offset)
    _rc(lib().dnni_las_write(os.fsencode(path), _ptr(xyz), _ptr(intensity), xyz.shape[0], sc, of),
        f"dnni_las_write {path}")


def write_asc(path, h, xll, yll, cellsize, nodata=-9999.0, nthreads=0):
    h = np.ascontiguousarray(h, np.float32)
    _rc(lib().dnni_write_asc(os.fsencode(path), _ptr(h), h.shape[1], h.shape[0], float(xll), float(yll),
                             float(cellsize), float(nodata), int(nthreads)), f"dnni_write_asc {path}")


def write_grid_bin(path, h, xll, yll, cellsize, nodata=-9999.0):
    h = np.ascontiguousarray(h, np.float32)
    _rc(lib().dnni_write_grid_bin(os.fsencode(path), _ptr(h), h.shape[1], h.shape[0], float(xll), float(yll),
                                  float(cellsize), float(nodata)), f"dnni_write_grid_bin {path}")
