"""The entry point that allocates nothing (dnni_interpolate_segment_device_noalloc).

It serves callers that cannot let a library call cudaMalloc/cudaFree (hosts
that own all device memory, latency-critical callers that cannot take the
implicit synchronisation): its scratch is a fixed 32 MiB device array inside
the library.  These tests call it through the C ABI and require bit-identical
heights and site maps to the allocating entry point
(dnni_interpolate_segment_device), on two calls in a row, so that the second
call also shows that leftovers of the first call in the shared array do not
leak into its result.  The file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from conftest import terrain_case

pytestmark = pytest.mark.gpu


def _noalloc(wp, d_xyz, n, d_h, d_site, stream):
    from terranni_b200 import engine
    return engine.lib().dnni_interpolate_segment_device_noalloc(
        ctypes.byref(wp), d_xyz.data_ptr() if d_xyz is not None else None, None, int(n), d_h.data_ptr(),
        d_site.data_ptr() if d_site is not None else None, stream)


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    from terranni_b200 import engine
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    cases = [
        (terrain_case(31, 300, 60000, lakes=2, lake_r=(10.0, 60.0)), engine.make_wp(300, 300, 100)),
        (terrain_case(32, 256, 9000, lakes=3, lake_r=(8.0, 50.0)),
         engine.make_wp(240, 250, 100, raster=(-6, -4, 250, 260), z_offset=12.5)),
    ]
    with engine.Engine(device=0) as eng:
        for xyz, wp in cases:           # two calls in a row, different sizes
            n = xyz.shape[0]
            d_xyz = torch.from_numpy(xyz).cuda()
            x0, y0, x1, y1 = engine.raster_box(wp)
            ref_h = torch.empty((wp.nrows, wp.ncols), dtype=torch.float32, device="cuda")
            ref_s = torch.empty((y1 - y0, x1 - x0), dtype=torch.int32, device="cuda")
            eng.interpolate_device(wp, d_xyz, n, ref_h, d_site=ref_s, stream=stream)
            h = torch.full((wp.nrows, wp.ncols), 123.0, dtype=torch.float32, device="cuda")
            s = torch.zeros((y1 - y0, x1 - x0), dtype=torch.int32, device="cuda")
            assert _noalloc(wp, d_xyz, n, h, s, stream) == 0
            torch.cuda.synchronize()
            assert torch.equal(h.view(torch.int32), ref_h.view(torch.int32))
            assert torch.equal(s, ref_s)


def test_noalloc_rejects_work_packages_beyond_its_scratch():
    import torch
    from terranni_b200 import engine
    torch.cuda.set_device(0)
    wp = engine.make_wp(4096, 4096, 100)
    d_xyz = torch.zeros((1, 3), dtype=torch.int32, device="cuda")
    d_h = torch.empty((4096, 4096), dtype=torch.float32, device="cuda")
    assert _noalloc(wp, d_xyz, 1, d_h, None, torch.cuda.current_stream().cuda_stream) == 10   # DNNI_E_SCRATCH
