"""The engine's search and packing code, built for the host (tests/native),
against the oracle: bit-exact site maps and heights on seeded cases that
exercise every search level, both accumulator forms and every stencil radius.
Runs on CPU; the same code runs on the GPU in test_gpu_parity.py."""
import numpy as np
import pytest

from conftest import golden_wp, load_golden, terrain_case

GOLDEN = load_golden()


def _same(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_host_build_matches_golden(emu, oracle, case):
    wp = golden_wp(oracle, case)
    for rs in (1, 3, 6):
        rc, r = emu(wp, case["xyz"], case["gid"], small_radius=rs)
        assert rc == 0
        assert np.array_equal(r["site"], case["site"])
        assert _same(r["h"], case["h"]), case["name"]


@pytest.mark.parametrize("seed,side,n,lakes,rs,bt", [
    (1, 96, 9000, 2, 3, 0),
    (2, 128, 20000, 3, 1, 0),
    (3, 80, 300, 1, 3, 0),        # sparse: large discs everywhere
    (4, 120, 15000, 2, 6, 1),
    (5, 100, 12000, 2, 2, 64),    # coarse bins
    (6, 64, 40, 0, 3, 0),         # very sparse
    (7, 140, 30000, 4, 4, 8),
])
def test_host_build_matches_oracle(emu, oracle, seed, side, n, lakes, rs, bt):
    xyz = terrain_case(seed, side, n, lakes=lakes, lake_r=(8.0, 30.0))
    wp = oracle.make_wp(side, side, 100)
    ref = oracle.interpolate(wp, xyz)
    rc, r = emu(wp, xyz, small_radius=rs, bin_target=bt)
    assert rc == 0
    assert np.array_equal(r["site"], ref["site"])
    assert _same(r["h"], ref["h"])


def test_host_build_raster_halo_and_origin(emu, oracle):
    rng = np.random.default_rng(12)
    n = 5000
    xyz = np.stack([rng.integers(-3000, 11000, n) + 500000, rng.integers(-2000, 9000, n) + 400000,
                    rng.integers(0, 30000, n)], 1).astype(np.int32)
    wp = oracle.make_wp(80, 70, 100, origin_x=500000, origin_y=400000, raster=(-12, -9, 95, 81),
                        z_scale=0.01, z_offset=123.0)
    ref = oracle.interpolate(wp, xyz)
    rc, r = emu(wp, xyz)
    assert rc == 0 and np.array_equal(r["site"], ref["site"]) and _same(r["h"], ref["h"])


def test_host_build_unpacked_accumulator(emu, oracle):
    # a handful of points with a huge z range: the packed word cannot hold the
    # per-cell sums, so the separate int64/int32 accumulators are used
    xyz = np.array([[0, 0, -900000000], [25500, 25500, 900000000], [12000, 300, 5]], np.int32)
    wp = oracle.make_wp(256, 256, 100)
    ref = oracle.interpolate(wp, xyz)
    rc, r = emu(wp, xyz)
    assert rc == 0 and r["info"]["packed"] == 0
    assert np.array_equal(r["site"], ref["site"]) and _same(r["h"], ref["h"])


def test_host_build_packed_when_it_fits(emu, oracle):
    xyz = terrain_case(9, 64, 3000, lakes=1, lake_r=(6.0, 12.0))
    rc, r = emu(oracle.make_wp(64, 64, 100), xyz)
    assert rc == 0 and r["info"]["packed"] == 1


def test_host_build_range_error(emu, oracle):
    xyz = np.array([[0, 0, 0], [2 ** 30 + 5, 0, 0]], np.int64).astype(np.int32)
    rc, _ = emu(oracle.make_wp(8, 8, 100), xyz)
    assert rc == 5   # DNNI_E_RANGE


def test_host_build_span_count_matches_oracle(emu, oracle):
    xyz = terrain_case(13, 90, 2500, lakes=2, lake_r=(8.0, 20.0))
    wp = oracle.make_wp(90, 90, 100)
    _, _, r2 = oracle.nearest(wp, xyz)
    rc, r = emu(wp, xyz, small_radius=3)
    big = r2 > 9
    assert r["info"]["big_pixels"] == int(big.sum())
    assert r["info"]["spans"] == int((2 * np.floor(np.sqrt(r2[big].astype(np.float64))) + 1).sum())


def _fallback_cases():
    rng = np.random.default_rng(77)
    # a dense cluster: a tile's bin window holds more points than shared memory
    dense = np.concatenate([
        np.stack([rng.integers(2000, 2600, 60000), rng.integers(3000, 3400, 60000), rng.integers(0, 9000, 60000)], 1),
        np.stack([rng.integers(0, 6400, 3000), rng.integers(0, 6400, 3000), rng.integers(0, 9000, 3000)], 1)])
    # cells much larger than bins: a tile's bin window has too many bins
    coarse = np.stack([rng.integers(0, 64 * 2000, 400000), rng.integers(0, 64 * 2000, 400000),
                       rng.integers(0, 9000, 400000)], 1)
    return [(dense.astype(np.int32), 64, 100, 0), (coarse.astype(np.int32), 64, 2000, 1)]


@pytest.mark.parametrize("k", [0, 1])
def test_host_build_window_fallbacks(emu, oracle, k):
    xyz, side, cs, bt = _fallback_cases()[k]
    wp = oracle.make_wp(side, side, cs)
    ref = oracle.interpolate(wp, xyz)
    rc, r = emu(wp, xyz, bin_target=bt)
    assert rc == 0 and np.array_equal(r["site"], ref["site"]) and _same(r["h"], ref["h"])


def test_cell_box_mask_matches_cell_by_cell(emu):
    # the seed of a far pixel takes the non-empty bins of square rings of a
    # block's 8 x 8 bins: every clipped range, including empty ones
    import ctypes, itertools, os
    L = ctypes.CDLL(os.path.join(os.path.dirname(__file__), "native", "libdnni_emu.so"))
    L.emu_cell_box_mask8.argtypes = [ctypes.c_int] * 4
    L.emu_cell_box_mask8.restype = ctypes.c_ulonglong
    for a0, a1, b0, b1 in itertools.product(range(-9, 17, 2), range(-3, 12), range(-9, 17, 2), range(-3, 12)):
        want = 0
        for y in range(8):
            for x in range(8):
                if a0 <= x <= a1 and b0 <= y <= b1:
                    want |= 1 << (8 * y + x)
        assert L.emu_cell_box_mask8(a0, a1, b0, b1) == want, (a0, a1, b0, b1)


def test_r2_of_is_exact_floor_division():
    import ctypes, os
    L = ctypes.CDLL(os.path.join(os.path.dirname(__file__), "native", "libdnni_emu.so"))
    L.emu_r2_of.argtypes = [ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int]
    L.emu_r2_of.restype = ctypes.c_int
    rng = np.random.default_rng(5)
    cap = 2 * 32767 * 32767
    for cs in (1, 7, 50, 100, 2000, 32767):
        cs2 = cs * cs
        for _ in range(2000):
            q = int(rng.integers(0, cap + 5))
            for d2 in (q * cs2 - 1, q * cs2, q * cs2 + cs2 - 1, int(rng.integers(0, 2 ** 62))):
                if d2 < 0:
                    continue
                assert L.emu_r2_of(d2, cs2, cap) == min(d2 // cs2, cap)
