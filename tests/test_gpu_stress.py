"""Point distributions at the extremes, bit-exact against the oracle: 20 000
points inside one cell (8 times a staged bin window; the fallback paths),
one point for a whole raster (every pixel goes to the far pass, discs span
the grid), points exactly on lattice positions (zero distances), and
collinear points (degenerate Voronoi cells)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.fixture(scope="module")
def eng():
    from terranni_b200 import engine
    e = engine.Engine(device=0)
    yield e
    e.close()


def _check(eng, oracle, ncols, nrows, cs, xyz, raster=None, gid=None):
    from terranni_b200 import engine
    args = {"raster": raster} if raster else {}
    ref = oracle.interpolate(oracle.make_wp(ncols, nrows, cs, **args), xyz, gid)
    h, site, _ = eng.interpolate(engine.make_wp(ncols, nrows, cs, **args), xyz, gid, site=True)
    assert np.array_equal(site, ref["site"])
    assert _same(h, ref["h"])
    return ref


def test_many_points_in_one_cell(eng, oracle):
    rng = np.random.default_rng(1)
    n = 20_000
    xyz = np.stack([12_800 + rng.integers(0, 100, n), 9_600 + rng.integers(0, 100, n),
                    rng.integers(0, 5000, n)], 1).astype(np.int32)
    ref = _check(eng, oracle, 256, 192, 100, xyz)
    assert (ref["C"] > 0).all()


def test_one_point_for_the_whole_raster(eng, oracle):
    ref = _check(eng, oracle, 512, 512, 100, np.array([[3_100, 47_700, 1234]], np.int32), raster=(-8, -8, 520, 520))
    assert np.all(ref["h"] == np.float32(12.34))


def test_points_on_the_lattice(eng, oracle):
    # every point exactly on a cell position: zero distances, R2 = 0 pixels,
    # and the rest of the lattice between them
    rng = np.random.default_rng(2)
    ij = rng.choice(300 * 200, 5000, replace=False)
    xyz = np.stack([(ij % 300) * 100, (ij // 300) * 100, rng.integers(-300, 300, 5000)], 1).astype(np.int32)
    gid = rng.permutation(5000).astype(np.uint32)
    _check(eng, oracle, 300, 200, 100, xyz, gid=gid)


def test_collinear_points(eng, oracle):
    # all sites on one diagonal line, many sharing positions: the Voronoi
    # cells are parallel strips with exact ties along their borders
    rng = np.random.default_rng(3)
    t = rng.integers(0, 180, 3000)
    xyz = np.stack([t * 100 + 50, t * 100 + 50, rng.integers(0, 1000, 3000)], 1).astype(np.int32)
    _check(eng, oracle, 200, 200, 100, xyz, raster=(-4, -4, 204, 204))


@pytest.mark.parametrize("raster", [(20, 15, 90, 60), (130, -40, 190, 10), (-60, 50, -5, 140)])
def test_rasters_that_do_not_cover_the_grid(eng, oracle, raster):
    # a raster inside the grid, and rasters beside it (cells take only the
    # discs that reach them; the rest are NODATA)
    rng = np.random.default_rng(sum(raster) & 0xFFFF)
    n = 6000 if raster[0] >= 0 and raster[2] <= 120 else 40     # sparse sites: discs reach the grid
    xyz = np.stack([rng.integers(-8000, 22000, n), rng.integers(-6000, 16000, n),
                    rng.integers(0, 3000, n)], 1).astype(np.int32)
    ref = _check(eng, oracle, 120, 100, 100, xyz, raster=raster)
    nod = (ref["h"] == np.float32(-9999.0)).mean()
    assert 0.0 < nod < 1.0
