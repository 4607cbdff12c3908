"""GPU parity: the CUDA engine (through its C ABI) against the golden
fixtures and the CPU oracle.  Integer work (site map, sums) is bit-exact, and
so are the float32 heights (one deterministic rounding chain); the stated
accuracy bar against FP64 is max |h - h_FP64| <= 1e-4 m."""
import numpy as np
import pytest

from conftest import golden_wp, load_golden, terrain_case

pytestmark = pytest.mark.gpu
GOLDEN = load_golden()
TOL_M = 1e-4


@pytest.fixture(scope="module")
def eng():
    from terranni_b200 import engine
    e = engine.Engine(device=0)
    yield e
    e.close()


def _same(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def _fp64_err(oracle, ref, h, wp):
    ok = ref["C"] > 0
    truth = oracle.exact_height_f64(ref["Z"][ok], ref["C"][ok], wp.z_scale, wp.z_offset)
    d = np.abs(h[ok].astype(np.float64) - truth)
    return float(d.max(initial=0.0)), float(np.sqrt(np.mean(d * d))) if d.size else 0.0


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_engine_matches_golden(eng, case):
    from terranni_b200 import engine
    wp = golden_wp(engine, case)
    h, site, st = eng.interpolate(wp, case["xyz"], case["gid"], site=True)
    assert np.array_equal(site, case["site"])
    assert _same(h, case["h"])


@pytest.mark.parametrize("seed,side,n,lakes,rs,bt", [
    (1, 96, 9000, 2, 3, 0),
    (2, 256, 60000, 3, 1, 0),
    (3, 200, 700, 1, 3, 0),
    (4, 300, 90000, 2, 6, 1),
    (5, 160, 30000, 2, 2, 64),
    (6, 64, 40, 0, 3, 0),
    (7, 384, 150000, 4, 4, 8),
])
def test_engine_matches_oracle(oracle, seed, side, n, lakes, rs, bt):
    from terranni_b200 import engine
    xyz = terrain_case(seed, side, n, lakes=lakes, lake_r=(8.0, 0.25 * side))
    wp = engine.make_wp(side, side, 100)
    ref = oracle.interpolate(oracle.make_wp(side, side, 100), xyz)
    with engine.Engine(device=0, small_radius=rs, bin_target=bt) as e:
        h, site, st = e.interpolate(wp, xyz, site=True)
    assert np.array_equal(site, ref["site"])
    assert _same(h, ref["h"])
    mx, rms = _fp64_err(oracle, ref, h, wp)
    assert mx <= TOL_M


def test_engine_raster_halo_origin_and_gid(eng, oracle):
    from terranni_b200 import engine
    rng = np.random.default_rng(12)
    n = 40000
    xyz = np.stack([rng.integers(-3000, 31000, n) + 500000, rng.integers(-2000, 27000, n) + 400000,
                    rng.integers(0, 30000, n)], 1).astype(np.int32)
    gid = rng.permutation(4 * n)[:n].astype(np.uint32)
    xyz[5, :2] = xyz[6, :2]
    args = dict(origin_x=500000, origin_y=400000, raster=(-17, -9, 290, 262), z_scale=0.01, z_offset=123.0)
    ref = oracle.interpolate(oracle.make_wp(280, 250, 100, **args), xyz, gid)
    h, site, _ = eng.interpolate(engine.make_wp(280, 250, 100, **args), xyz, gid, site=True)
    assert np.array_equal(site, ref["site"]) and _same(h, ref["h"])


def test_engine_unpacked_accumulator(eng, oracle):
    from terranni_b200 import engine
    xyz = np.array([[0, 0, -900000000], [25500, 25500, 900000000], [12000, 300, 5]], np.int32)
    ref = oracle.interpolate(oracle.make_wp(256, 256, 100), xyz)
    h, site, st = eng.interpolate(engine.make_wp(256, 256, 100), xyz, site=True)
    assert st.packed == 0
    assert np.array_equal(site, ref["site"]) and _same(h, ref["h"])


def test_engine_empty_and_errors(eng):
    from terranni_b200 import engine
    h, site, st = eng.interpolate(engine.make_wp(9, 4, 100, nodata=-7.0), np.zeros((0, 3), np.int32), site=True)
    assert np.all(h == np.float32(-7.0)) and np.all(site == engine.NO_SITE) and st.nodata_cells == 36
    with pytest.raises(engine.DnniError) as ei:
        eng.interpolate(engine.make_wp(8, 8, 100), np.array([[0, 0, 0], [2 ** 30 + 5, 0, 0]], np.int64).astype(np.int32))
    assert ei.value.status == 5
    with pytest.raises(engine.DnniError) as ei:
        eng.interpolate(engine.make_wp(0, 8, 100), np.zeros((1, 3), np.int32))
    assert ei.value.status == 1
    # the context stays usable after errors
    h, _, _ = eng.interpolate(engine.make_wp(4, 4, 100), np.array([[100, 100, 500]], np.int32))
    assert np.all(h == np.float32(5.0))


def test_engine_mem_budget_refuses(oracle):
    from terranni_b200 import engine
    with engine.Engine(device=0, mem_budget=1 << 20) as e:
        with pytest.raises(engine.DnniError) as ei:
            e.interpolate(engine.make_wp(1024, 1024, 100), np.zeros((1, 3), np.int32))
        assert ei.value.status == 2


def test_device_path_matches_host_path(eng):
    import torch
    from terranni_b200 import engine
    xyz = terrain_case(21, 512, 300000, lakes=3, lake_r=(10.0, 80.0))
    wp = engine.make_wp(512, 512, 100)
    h_host, site_host, _ = eng.interpolate(wp, xyz, site=True)
    d_xyz = torch.from_numpy(xyz).cuda()
    d_h = torch.empty((512, 512), dtype=torch.float32, device="cuda")
    d_site = torch.empty((512, 512), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = eng.interpolate_device(wp, d_xyz, xyz.shape[0], d_h, d_site=d_site, stream=stream)
    torch.cuda.synchronize()
    assert _same(d_h.cpu().numpy(), h_host)
    assert np.array_equal(d_site.cpu().numpy().view(np.uint32), site_host)
    assert st.n_points == xyz.shape[0] and st.ms_total > 0


def test_deterministic_and_order_independent(eng):
    from terranni_b200 import engine
    xyz = terrain_case(22, 600, 400000, lakes=4, lake_r=(20.0, 120.0))
    wp = engine.make_wp(600, 600, 100)
    h1, s1, _ = eng.interpolate(wp, xyz, site=True)
    # shuffled input order, each point keeping its original index as its id
    perm = np.random.default_rng(0).permutation(xyz.shape[0])
    h2, s2, _ = eng.interpolate(wp, xyz[perm], perm.astype(np.uint32), site=True)
    assert _same(h1, h2) and np.array_equal(s1, s2)
    h3, s3, _ = eng.interpolate(wp, xyz, site=True)
    assert _same(h1, h3) and np.array_equal(s1, s3)


def test_sinusoid_512_full_size(eng, oracle):
    """The 512 x 512 / 200k-point sinusoid workload at full size."""
    from terranni_b200 import engine, synth
    w = synth.config1()
    wp = engine.make_wp(512, 512, 100)
    ref = oracle.interpolate(oracle.make_wp(512, 512, 100), w["xyz"])
    h, site, st = eng.interpolate(wp, w["xyz"], site=True)
    assert np.array_equal(site, ref["site"]) and _same(h, ref["h"])
    mx, rms = _fp64_err(oracle, ref, h, wp)
    assert mx <= TOL_M and st.nodata_cells == 0


@pytest.mark.parametrize("k", [0, 1])
def test_engine_window_fallbacks(oracle, k):
    from terranni_b200 import engine
    from test_kernel_logic_host import _fallback_cases
    xyz, side, cs, bt = _fallback_cases()[k]
    ref = oracle.interpolate(oracle.make_wp(side, side, cs), xyz)
    with engine.Engine(device=0, bin_target=bt) as e:
        h, site, _ = e.interpolate(engine.make_wp(side, side, cs), xyz, site=True)
    assert np.array_equal(site, ref["site"]) and _same(h, ref["h"])


@pytest.mark.parametrize("kind", ["wide_z", "wide_discs"])
def test_span_path_extremes(eng, oracle, kind):
    """Extremes of the span path: a z range near the int32 limit (unpacked
    accumulators), and discs of up to 1700 cells (one site on a long grid)."""
    from terranni_b200 import engine
    rng = np.random.default_rng(9)
    if kind == "wide_z":
        side, n = 200, 3000
        xyz = terrain_case(12, side, n, lakes=2, lake_r=(10.0, 40.0))
        xyz[:, 2] = rng.integers(-400_000_000, 400_000_000, n, dtype=np.int64).astype(np.int32)
    else:                       # a thin grid with one site at its left end: radii up to 1700 cells
        side, n = 1700, 1
        xyz = np.array([[0, 1500, 777]], np.int32)
    rows = side if kind == "wide_z" else 40
    wp = engine.make_wp(side, rows, 100)
    ref = oracle.interpolate(oracle.make_wp(side, rows, 100), xyz)
    h, site, st = eng.interpolate(wp, xyz, site=True)
    assert np.array_equal(site, ref["site"])
    assert _same(h, ref["h"])
