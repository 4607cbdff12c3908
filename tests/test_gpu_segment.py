"""Segment driver (dnni_segment_run): one grid interpolated as tiles with
halos, from host memory.

Each tile's halo is checked after it runs and grown until no pixel outside
its raster can reach its cells and no point outside its point box can be
nearer than the site found, so the stitched grid must be bit-identical —
heights and site map, seams included — to one work package covering the
whole grid (raster = grid), which the other tests tie to the oracle."""
import numpy as np
import pytest

from conftest import terrain_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    import torch
    from terranni_b200 import engine
    torch.cuda.set_device(0)
    e = engine.Engine(device=0)
    yield e
    e.close()


def _cloud(seed, ncols, nrows, n, cell=100, margin=30, lakes=3):
    """Terrain points over the grid plus a margin of cells on every side."""
    side = max(ncols, nrows) + 2 * margin
    xyz = terrain_case(seed, side, n, cell=cell, lakes=lakes, lake_r=(0.02 * side, 0.12 * side))
    xyz = xyz - np.array([margin * cell, margin * cell, 0], np.int32)
    return xyz


@pytest.mark.parametrize("ncols,nrows,tile,halo,tpb,n,lakes", [
    (1100, 900, 256, 8, 4, 500_000, 3),     # halos start too small: reruns
    (700, 650, 200, 64, 1, 150_000, 2),     # odd tiles, one per batch
    (500, 300, 512, 4, 16, 20_000, 4),      # one tile row, sparse points
    (1300, 1000, 256, 0, 8, 400_000, 4),    # halos from the occupancy bound
])
def test_segment_equals_one_work_package(eng, ncols, nrows, tile, halo, tpb, n, lakes):
    from terranni_b200 import engine
    ox, oy = 50_000_000, 400_000_000
    xyz = _cloud(7 + ncols, ncols, nrows, n, lakes=lakes) + np.array([ox, oy, 0], np.int32)
    ref_h, ref_s, _ = eng.interpolate(engine.make_wp(ncols, nrows, 100, ox, oy), xyz, site=True)
    h, s, st = eng.segment_run(xyz, ncols, nrows, 100, origin=(ox, oy), tile=tile, halo=halo, tiles_per_batch=tpb,
                               site=True)
    assert np.array_equal(s, ref_s)
    assert np.array_equal(h.view(np.uint32), ref_h.view(np.uint32))
    ntile = -(-ncols // tile) * -(-nrows // tile)
    assert st.tiles == ntile and st.tile_runs >= ntile and st.max_halo >= halo
    if halo == 0:                            # the bound is an upper bound: no reruns
        assert st.tile_runs == ntile
    assert st.points == xyz.shape[0] and st.cells == ncols * nrows


def test_segment_mosaic_against_the_oracle(eng, oracle):
    # the stitched grid checked directly against the oracle's one work
    # package: site map and heights bit for bit, FP64 error within 1e-4 m
    ncols, nrows = 900, 700
    ox, oy = 12_000_000, 34_000_000
    xyz = _cloud(41, ncols, nrows, 200_000, lakes=3) + np.array([ox, oy, 0], np.int32)
    h, s, st = eng.segment_run(xyz, ncols, nrows, 100, origin=(ox, oy), tile=256, halo=0, tiles_per_batch=4,
                               site=True)
    ref = oracle.interpolate(oracle.make_wp(ncols, nrows, 100, ox, oy), xyz)
    assert np.array_equal(s, ref["site"])
    assert np.array_equal(h.view(np.uint32), ref["h"].view(np.uint32))
    ok = ref["C"] > 0
    truth = oracle.exact_height_f64(ref["Z"][ok], ref["C"][ok], 0.01, 0.0)
    assert np.abs(h[ok].astype(np.float64) - truth).max() <= 1e-4
    assert st.tiles == 12


@pytest.mark.parametrize("parts", [2, 3])
def test_segment_parts_stitch_to_the_whole_grid(eng, parts):
    # each part's call (here one after another on one GPU; in a multi-GPU
    # run, one per rank) writes only its own tiles' cells; together the parts
    # give the whole grid bit for bit, every tile run by exactly one part
    ncols, nrows = 1000, 760
    xyz = _cloud(19, ncols, nrows, 250_000, lakes=3)
    whole, _, st_all = eng.segment_run(xyz, ncols, nrows, 100, tile=200, halo=0, tiles_per_batch=4)
    h = np.full((nrows, ncols), np.nan, np.float32)
    tiles = 0
    for p in range(parts):
        before = np.isnan(h).sum()
        _, _, st = eng.segment_run(xyz, ncols, nrows, 100, tile=200, halo=0, tiles_per_batch=4, out_h=h,
                                   part=p, parts=parts)
        assert st.tiles > 0 and np.isnan(h).sum() < before
        if p < parts - 1:
            assert np.isnan(h).any()
        tiles += st.tiles
    assert tiles == st_all.tiles == 5 * 4
    assert np.array_equal(h.view(np.uint32), whole.view(np.uint32))


def test_segment_reruns_tiles_whose_halo_is_too_small(eng):
    ncols = nrows = 600
    xyz = _cloud(3, ncols, nrows, 40_000, lakes=4)
    _, _, st = eng.segment_run(xyz, ncols, nrows, 100, tile=128, halo=2)
    assert st.tile_runs > st.tiles and st.max_halo > 2


def test_segment_without_points_is_all_nodata(eng):
    h, s, st = eng.segment_run(np.zeros((0, 3), np.int32), 300, 200, 100, tile=128, site=True)
    assert np.all(h == np.float32(-9999.0)) and np.all(s == 0xFFFFFFFF)
    assert st.tile_runs == st.tiles


@pytest.mark.parametrize("npts,halo", [(1, 0), (3, 0), (5, 4)])
def test_segment_with_a_few_points_for_the_whole_grid(eng, npts, halo):
    # the occupancy bound makes halos of hundreds of cells (or, from a small
    # first halo, reruns grow them); the grid must still equal one work package
    from terranni_b200 import engine
    rng = np.random.default_rng(npts)
    xyz = np.stack([rng.integers(0, 60_000, npts), rng.integers(0, 40_000, npts),
                    rng.integers(0, 9000, npts)], 1).astype(np.int32)
    ref_h, ref_s, _ = eng.interpolate(engine.make_wp(600, 400, 100), xyz, site=True)
    h, s, st = eng.segment_run(xyz, 600, 400, 100, tile=128, halo=halo, tiles_per_batch=8, site=True)
    assert np.array_equal(s, ref_s)
    assert np.array_equal(h.view(np.uint32), ref_h.view(np.uint32))
    assert st.max_halo > 100


def test_segment_with_all_points_beyond_the_grid(eng):
    # the points lie 2-3 km west of and below the grid: they fall into the
    # edge buckets, the occupancy bound underestimates their distance, and
    # the halo checks must grow the boxes until the stitched grid equals one
    # work package
    from terranni_b200 import engine
    rng = np.random.default_rng(9)
    xyz = np.stack([rng.integers(-300_000, -200_000, 30), rng.integers(-250_000, 40_000, 30),
                    rng.integers(0, 9000, 30)], 1).astype(np.int32)
    ref_h, ref_s, _ = eng.interpolate(engine.make_wp(400, 300, 100), xyz, site=True)
    h, s, st = eng.segment_run(xyz, 400, 300, 100, tile=128, halo=0, tiles_per_batch=4, site=True)
    assert np.array_equal(s, ref_s)
    assert np.array_equal(h.view(np.uint32), ref_h.view(np.uint32))
