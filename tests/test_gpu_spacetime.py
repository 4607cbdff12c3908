"""Space-time interpolation on the GPU (dnni_interpolate_spacetime, the
timeRadius > 0 path of nni::performNNI, nni.cpp:902-933): heights bit-exact
against the oracle's restatement over slices, lifted time distances and
slice-lifted queries; time radius 0 equal to the 2-D call; edge cases."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from terranni_b200 import engine
    e = engine.Engine(device=0)
    yield e
    e.close()


def _terrain(seed, side, n, cs, cur, rt, spread):
    from conftest import terrain_case
    xyz = terrain_case(seed, side, n, lakes=1, lake_r=(5.0, 15.0)).astype(np.int64)
    xyz[:, :2] = xyz[:, :2] * cs // 100
    rng = np.random.default_rng(seed)
    t = rng.integers(cur - spread, cur + spread + 1, xyz.shape[0]).astype(np.int32)
    return xyz.astype(np.int32), t


@pytest.mark.parametrize("rt,tau,side,n,raster", [(1, 100, 96, 4000, None), (2, 50, 128, 9000, 4),
                                                    (3, 1000, 80, 3000, 2), (2, 1, 64, 2500, None)])
def test_spacetime_matches_oracle(eng, oracle, rt, tau, side, n, raster):
    from terranni_b200 import engine
    cur = 10
    xyz, t = _terrain(7 + rt, side, n, 100, cur, rt, 3 * rt + 1)
    xyz[5, :2] = xyz[4, :2]                     # a tie on position and time
    t[5] = t[4]
    args = {"raster": (-raster, -raster, side + raster, side + raster)} if raster else {}
    wp_o = oracle.make_wp(side, side, 100, **args)
    wp_e = engine.make_wp(side, side, 100, **args)
    ref = oracle.interpolate_spacetime(wp_o, xyz, t, cur, rt, tau)
    h, st = eng.interpolate_spacetime(wp_e, xyz, t, cur, rt, tau)
    assert np.array_equal(h.view(np.uint32), ref["h"].view(np.uint32))
    assert st.n_pixels == (2 * rt + 1) * wp_pixels(wp_e) and st.ms_total > 0
    assert (ref["h"] != np.float32(-9999.0)).mean() > 0.9


def wp_pixels(wp):
    from terranni_b200 import engine
    x0, y0, x1, y1 = engine.raster_box(wp)
    return (x1 - x0) * (y1 - y0)


def test_spacetime_radius_zero_is_the_2d_call(eng):
    from terranni_b200 import engine
    xyz, t = _terrain(3, 200, 20000, 100, 4, 2, 3)
    wp = engine.make_wp(200, 200, 100, raster=(-3, -3, 203, 203))
    h, _ = eng.interpolate_spacetime(wp, xyz, t, 4, 0, 100)
    sel = t == 4
    h2, _, _ = eng.interpolate(wp, xyz[sel])
    assert np.array_equal(h.view(np.uint32), h2.view(np.uint32))


def test_spacetime_gaps_empty_and_errors(eng, oracle):
    from terranni_b200 import engine
    xyz, t = _terrain(11, 64, 2000, 100, 0, 2, 6)
    t[(t == -1) | (t == 1)] = 7                  # slices with no site of their own
    wp_e, wp_o = engine.make_wp(64, 64, 100), oracle.make_wp(64, 64, 100)
    h, _ = eng.interpolate_spacetime(wp_e, xyz, t, 0, 2, 100)
    ref = oracle.interpolate_spacetime(wp_o, xyz, t, 0, 2, 100)
    assert np.array_equal(h.view(np.uint32), ref["h"].view(np.uint32))
    h, _ = eng.interpolate_spacetime(wp_e, np.zeros((0, 3), np.int32), np.zeros(0, np.int32), 0, 1, 100)
    assert np.all(h == np.float32(-9999.0))
    h, _ = eng.interpolate_spacetime(wp_e, xyz, np.full(xyz.shape[0], 50, np.int32), 0, 1, 100)
    assert np.all(h == np.float32(-9999.0))                 # nothing within reach of time 0
    for rt, tau in ((17, 100), (1, 0), (4, 1 << 29)):
        with pytest.raises(engine.DnniError) as ei:
            eng.interpolate_spacetime(wp_e, xyz, t, 0, rt, tau)
        assert ei.value.status == 1


def test_spacetime_constant_field_at_size(eng):
    # a 2048 x 2048 grid, 2 M points over 9 time values: a constant z stays constant
    from terranni_b200 import engine
    rng = np.random.default_rng(5)
    n = 2_000_000
    xyz = np.stack([rng.integers(0, 204800, n), rng.integers(0, 204800, n), np.full(n, 1234)], 1).astype(np.int32)
    t = rng.integers(96, 105, n).astype(np.int32)
    h, st = eng.interpolate_spacetime(engine.make_wp(2048, 2048, 100), xyz, t, 100, 2, 100)
    assert np.all(h == np.float32(12.34)) and st.nodata_cells == 0


def test_spacetime_negative_times_and_origin(eng, oracle):
    # times below zero, the current time negative, a work package away from
    # the LAS origin with a raster halo
    from terranni_b200 import engine
    xyz, t = _terrain(31, 72, 3000, 100, -3, 1, 4)
    xyz[:, 0] += 123400
    xyz[:, 1] -= 56700
    args = dict(origin_x=123400, origin_y=-56700, raster=(-3, -3, 75, 75))
    ref = oracle.interpolate_spacetime(oracle.make_wp(72, 72, 100, **args), xyz, t, -3, 1, 100)
    h, _ = eng.interpolate_spacetime(engine.make_wp(72, 72, 100, **args), xyz, t, -3, 1, 100)
    assert np.array_equal(h.view(np.uint32), ref["h"].view(np.uint32))
    assert (ref["h"] != np.float32(-9999.0)).mean() > 0.9


def test_spacetime_device_buffers_equal_host_buffers(eng):
    # dnni_interpolate_spacetime_device: the same heights from device-resident
    # points and times, read back after the call queued on torch's stream
    import torch
    from terranni_b200 import engine
    xyz, t = _terrain(41, 160, 12000, 100, 8, 2, 6)
    wp = engine.make_wp(160, 160, 100, raster=(-3, -3, 163, 163))
    h_host, _ = eng.interpolate_spacetime(wp, xyz, t, 8, 2, 100)
    d_xyz = torch.from_numpy(xyz).cuda()
    d_t = torch.from_numpy(t).cuda()
    for stats in (True, False):
        d_h = torch.zeros(160 * 160, dtype=torch.float32, device="cuda")
        eng.interpolate_spacetime_device(wp, d_xyz, d_t, xyz.shape[0], d_h, 8, 2, 100,
                                         stream=torch.cuda.current_stream().cuda_stream, stats=stats)
        h = d_h.cpu().numpy().reshape(160, 160)
        assert np.array_equal(h.view(np.uint32), h_host.view(np.uint32))


def test_spacetime_largest_time_radius(eng, oracle):
    # time radius 16: 33 slices over 65 time values (the largest parameter
    # block and batch of the space-time path)
    from terranni_b200 import engine
    rng = np.random.default_rng(16)
    n = 5000
    xyz = np.stack([rng.integers(0, 4800, n), rng.integers(0, 4000, n), rng.integers(0, 9000, n)], 1).astype(np.int32)
    t = rng.integers(-40, 41, n).astype(np.int32)
    wp_o = oracle.make_wp(48, 40, 100, raster=(-2, -2, 50, 42))
    wp_e = engine.make_wp(48, 40, 100, raster=(-2, -2, 50, 42))
    ref = oracle.interpolate_spacetime(wp_o, xyz, t, 0, 16, 25)
    h, st = eng.interpolate_spacetime(wp_e, xyz, t, 0, 16, 25)
    assert np.array_equal(h.view(np.uint32), ref["h"].view(np.uint32))
    assert st.n_pixels == 33 * 52 * 44
