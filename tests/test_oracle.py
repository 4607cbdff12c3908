"""CPU oracle: pinned against the golden known answers and brute force."""
import numpy as np
import pytest

from conftest import golden_wp, load_golden

GOLDEN = load_golden()


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_oracle_matches_golden(oracle, case):
    wp = golden_wp(oracle, case)
    for brute in (False, True):
        r = oracle.interpolate(wp, case["xyz"], case["gid"], brute=brute)
        assert np.array_equal(r["site"], case["site"])
        assert np.array_equal(r["Z"], case["Z"]) and np.array_equal(r["C"], case["C"])
        assert np.array_equal(r["h"].view(np.uint32), case["h"].view(np.uint32))


def test_oracle_random_vs_brute(oracle):
    rng = np.random.default_rng(7)
    for trial in range(40):
        nc, nr = (int(v) for v in rng.integers(1, 24, 2))
        cs = int(rng.choice([1, 7, 50, 100]))
        n = int(rng.integers(0, 60))
        xyz = np.stack([rng.integers(-3 * cs, (nc + 3) * cs, n), rng.integers(-3 * cs, (nr + 3) * cs, n),
                        rng.integers(-500, 500, n)], 1).astype(np.int32)
        if n > 3 and trial % 3 == 0:
            xyz[1, :2] = xyz[0, :2]
            xyz[2, :2] = xyz[0, :2]
        raster = (-2, -1, nc + 3, nr + 2) if trial % 2 else None
        gid = rng.permutation(10 * n + 1)[:n].astype(np.uint32) if trial % 4 == 1 else None
        wp = oracle.make_wp(nc, nr, cs, raster=raster)
        a = oracle.interpolate(wp, xyz, gid)
        b = oracle.interpolate(wp, xyz, gid, brute=True)
        assert np.array_equal(a["site"], b["site"])
        assert np.array_equal(a["Z"], b["Z"]) and np.array_equal(a["C"], b["C"])
        assert np.array_equal(a["h"].view(np.uint32), b["h"].view(np.uint32))


def test_single_site_everywhere(oracle):
    wp = oracle.make_wp(33, 21, 100)
    r = oracle.interpolate(wp, np.array([[1234, 567, 4321]]))
    assert (r["C"] >= 1).all()
    assert np.all(r["h"] == np.float32(4321 * 0.01))


def test_constant_field_is_constant(oracle):
    rng = np.random.default_rng(3)
    xyz = np.stack([rng.integers(0, 6400, 500), rng.integers(0, 4800, 500), np.full(500, 777)], 1)
    r = oracle.interpolate(oracle.make_wp(64, 48, 100), xyz)
    assert np.all(r["h"] == np.float32(7.77))


def test_mirror_symmetry(oracle):
    # two sites mirrored about the grid's vertical axis (x = 950, between two
    # lattice columns, so no pixel is equidistant) with swapped z: the output
    # mirrors
    wp = oracle.make_wp(20, 9, 100)
    a = oracle.interpolate(wp, np.array([[530, 410, 100], [1370, 410, 900]]))
    b = oracle.interpolate(wp, np.array([[530, 410, 900], [1370, 410, 100]]))
    assert np.array_equal(a["Z"], b["Z"][:, ::-1]) and np.array_equal(a["C"], b["C"][:, ::-1])


def test_lowest_gid_wins_ties(oracle):
    xyz = np.array([[250, 250, 1], [250, 250, 2], [250, 250, 3]])
    gid = np.array([9, 4, 6], np.uint32)
    sg, sz, _ = oracle.nearest(oracle.make_wp(5, 5, 100), xyz, gid)
    assert np.all(sg == 4) and np.all(sz == 2)


def test_empty_is_nodata(oracle):
    r = oracle.interpolate(oracle.make_wp(7, 3, 100, nodata=-1.5), np.zeros((0, 3), np.int32))
    assert np.all(r["h"] == np.float32(-1.5)) and np.all(r["site"] == oracle.NO_SITE)


def test_invalid_workpackage(oracle):
    with pytest.raises(ValueError):
        oracle.interpolate(oracle.make_wp(0, 3, 100), np.zeros((1, 3), np.int32))
    with pytest.raises(ValueError):
        oracle.interpolate(oracle.make_wp(4, 3, 100, raster=(2, 2, 1, 5)), np.zeros((1, 3), np.int32))


def test_compat_multiplier_formula(oracle):
    # terranni.cpp:675-684 at CLI defaults (site radius 5, scaling 5, cell 2)
    import math
    for zmax, pmin in ((300.0, 0), (1234.5, -12), (10.0, 3)):
        pw = math.ceil(2.0 * 5.0 * 5 / 2.0)
        m = int(math.floor(2147483647 / (pw * pw * (zmax - pmin))))
        m = int(10 ** math.floor(math.log10(m)))
        assert oracle.compat_multiplier(5.0, 5, 2.0, zmax, pmin) == m


def test_compat_emulation_smoke(oracle):
    s = oracle.CompatSettings(scale=5, cell_size=2.0, site_radius=5.0, query_radius=5 * 2.0 / 2 - 0.01,
                              point_min=0, multiplier=10000, total_ncols=40, total_nrows=30)
    cwp = oracle.CompatWP(origin_x=0.0, origin_y=0.0, grid_origin_x=0.0, grid_origin_y=0.0, nrows=30, ncols=40)
    rng = np.random.default_rng(5)
    pts = np.stack([rng.uniform(0, 80, 3000), rng.uniform(0, 60, 3000), rng.uniform(10, 20, 3000)], 1)
    h, res = oracle.compat(s, cwp, pts)
    ok = h != -9999
    assert ok.mean() > 0.95
    assert h[ok].min() >= 9.0 - 1e-3 and h[ok].max() <= 20.0 + 1e-3


def test_gl_disagreement_is_a_fraction(oracle):
    rng = np.random.default_rng(11)
    xyz = np.stack([rng.integers(0, 6400, 4000), rng.integers(0, 6400, 4000), rng.integers(0, 9000, 4000)], 1)
    d = oracle.gl_disagreement(oracle.make_wp(64, 64, 100), xyz)
    assert d["pixels"] == 64 * 64
    assert 0.0 <= d["site_frac"] <= 1.0 and d["z_differs"] <= d["site_differs"]


def _st_case(rng, n, nc, nr, cs, cur, rt):
    xyz = np.stack([rng.integers(-3 * cs, (nc + 3) * cs, n), rng.integers(-3 * cs, (nr + 3) * cs, n),
                    rng.integers(-500, 500, n)], 1).astype(np.int32)
    t = rng.integers(cur - 3 * rt - 1, cur + 3 * rt + 2, n).astype(np.int32)
    return xyz, t


def test_spacetime_kd_matches_brute(oracle):
    # the per-time-value k-d form against every point for every (slice, pixel)
    rng = np.random.default_rng(1)
    for trial in range(40):
        nc, nr = (int(v) for v in rng.integers(1, 20, 2))
        cs = int(rng.choice([1, 7, 100]))
        rt, tau, cur = int(rng.integers(0, 4)), int(rng.choice([1, 50, 100, 1000])), int(rng.integers(-3, 10))
        xyz, t = _st_case(rng, int(rng.integers(0, 50)), nc, nr, cs, cur, rt)
        if xyz.shape[0] > 3:
            xyz[1, :2] = xyz[0, :2]
            t[1] = t[0]
        wp = oracle.make_wp(nc, nr, cs, raster=(-2, -1, nc + 3, nr + 2) if trial % 2 else None)
        a = oracle.interpolate_spacetime(wp, xyz, t, cur, rt, tau)
        b = oracle.interpolate_spacetime(wp, xyz, t, cur, rt, tau, brute=True)
        assert np.array_equal(a["Z"], b["Z"]) and np.array_equal(a["C"], b["C"])
        assert np.array_equal(a["h"].view(np.uint32), b["h"].view(np.uint32))


def test_spacetime_radius_zero_is_the_2d_slice(oracle):
    rng = np.random.default_rng(2)
    xyz, t = _st_case(rng, 400, 30, 25, 100, 5, 2)
    wp = oracle.make_wp(30, 25, 100, raster=(-3, -3, 33, 28))
    a = oracle.interpolate_spacetime(wp, xyz, t, 5, 0, 100)
    sel = t == 5
    b = oracle.interpolate(wp, xyz[sel], np.nonzero(sel)[0].astype(np.uint32))
    assert np.array_equal(a["Z"], b["Z"]) and np.array_equal(a["C"], b["C"])


def test_spacetime_known_answers(oracle):
    rng = np.random.default_rng(3)
    wp = oracle.make_wp(24, 18, 100)
    # a constant field stays constant whatever the times
    xyz = np.stack([rng.integers(0, 2400, 300), rng.integers(0, 1800, 300), np.full(300, 4321)], 1)
    t = rng.integers(0, 9, 300)
    assert np.all(oracle.interpolate_spacetime(wp, xyz, t, 4, 2, 100)["h"] == np.float32(43.21))
    # one site: every slice within reach sees it; the slice it is in covers every cell
    r = oracle.interpolate_spacetime(wp, np.array([[1200, 900, 777]]), np.array([5]), 4, 2, 100)
    assert np.all(r["h"] == np.float32(7.77)) and np.all(r["C"] >= 1)
    # points farther than 2 rt from the current time take part in no slice
    far = np.concatenate([xyz, [[1200, 900, 99999]]])
    tf = np.concatenate([t, [4 + 5]])
    assert np.array_equal(oracle.interpolate_spacetime(wp, far, tf, 4, 2, 100)["Z"],
                          oracle.interpolate_spacetime(wp, xyz, t, 4, 2, 100)["Z"])
    # a slice with no site leaves nothing; no points at all: nodata
    e = oracle.interpolate_spacetime(wp, np.zeros((0, 3), np.int32), np.zeros(0, np.int32), 0, 1, 100)
    assert np.all(e["h"] == np.float32(-9999.0)) and np.all(e["C"] == 0)
    with pytest.raises(ValueError):
        oracle.interpolate_spacetime(wp, xyz, t, 4, 17, 100)
