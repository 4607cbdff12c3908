"""The reference's only data fixture, data-generator.py, restated.

Its space-time scenario is a wall moving through a flat field
(data-generator.py:30-41: height 20 inside a 5 m wide strip whose left edge
moves from xmin to xmax as t goes from 0 to 100, height 1 elsewhere), points
uniform on [-100, 100]^2 at a 0.001 m granularity (data-generator.py:49-54,
80), at times 0..109 with 10, 30, 50, 70 and 90 left out (data-generator.py:
90-95) -- the missing slices are what space-time interpolation fills in.

Known answers: at a missing time, every cell farther than the reach of the
neighbouring slices' walls takes exactly the flat height; cells inside the
wall's path interpolate between the two.  The oracle is checked on that
here, and the GPU against the oracle bit for bit (gpu)."""
import numpy as np
import pytest

XY = 0.001            # LAS units of the fixture's 0.001 m granularity
Z = 0.01


def wall_points(times, n_per_time, seed):
    rng = np.random.default_rng(seed)
    xs, ys, zs, ts = [], [], [], []
    for t in times:
        x = rng.integers(-100000, 100000, n_per_time)
        y = rng.integers(-100000, 100000, n_per_time)
        xm = (t / 100.0) * 200.0 - 100.0                     # the strip's left edge, metres
        inside = (x * XY >= xm) & (x * XY < xm + 5.0)
        xs.append(x)
        ys.append(y)
        zs.append(np.where(inside, 2000, 100))               # 20 m / 1 m in 0.01 m units
        ts.append(np.full(n_per_time, t))
    xyz = np.stack([np.concatenate(xs), np.concatenate(ys), np.concatenate(zs)], 1).astype(np.int32)
    return xyz, np.concatenate(ts).astype(np.int32)


def fixture_case(oracle_or_engine, cur=50, rt=1, n_per_time=6000):
    times = [t for t in range(40, 61) if t not in (10, 30, 50, 70, 90)]
    xyz, t = wall_points(times, n_per_time, 1234)
    # 200 x 200 cells of 1 m over the fixture's square
    wp = oracle_or_engine.make_wp(200, 200, 1000, origin_x=-100000, origin_y=-100000, z_scale=Z)
    return wp, xyz, t, cur, rt


def far_from_walls(cur, rt, margin_m):
    # the walls of every time that can reach the slices of cur (|t - cur| <= 2 rt)
    lo = (cur - 2 * rt) / 100.0 * 200.0 - 100.0
    hi = (cur + 2 * rt) / 100.0 * 200.0 - 100.0 + 5.0
    xc = -100.0 + np.arange(200) * 1.0                        # cell centres (lattice points), metres
    return (xc < lo - margin_m) | (xc >= hi + margin_m)


def test_missing_slice_is_filled_from_its_neighbours(oracle):
    wp, xyz, t, cur, rt = fixture_case(oracle)
    assert not np.any(t == cur)                               # time 50 has no points of its own
    r = oracle.interpolate_spacetime(wp, xyz, t, cur, rt, 1000)
    h = r["h"]
    assert np.all(r["C"] > 0)
    cols = far_from_walls(cur, rt, 15.0)
    assert np.all(h[:, cols] == np.float32(1.0))             # the flat field, exactly
    wall = (np.arange(200) - 100.0 >= 0.0) & (np.arange(200) - 100.0 < 5.0)
    assert h[:, wall].mean() > 5.0                            # the wall's path is lifted
    assert h.max() <= np.float32(20.0) and h.min() >= np.float32(1.0)


def test_time_radius_zero_at_a_missing_slice_is_nodata(oracle):
    wp, xyz, t, cur, _ = fixture_case(oracle)
    r = oracle.interpolate_spacetime(wp, xyz, t, cur, 0, 1000)
    assert np.all(r["h"] == np.float32(-9999.0))


@pytest.mark.gpu
@pytest.mark.parametrize("cur,rt", [(50, 1), (50, 2), (47, 1)])
def test_wall_fixture_gpu_matches_oracle(oracle, cur, rt):
    from terranni_b200 import engine
    wpo, xyz, t, _, _ = fixture_case(oracle, cur, rt)
    wpe, _, _, _, _ = fixture_case(engine, cur, rt)
    ref = oracle.interpolate_spacetime(wpo, xyz, t, cur, rt, 1000)
    with engine.Engine(device=0) as e:
        h, _ = e.interpolate_spacetime(wpe, xyz, t, cur, rt, 1000)
    assert np.array_equal(h.view(np.uint32), ref["h"].view(np.uint32))
