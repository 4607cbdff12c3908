"""Batched execution (dnni_batch_*): many work packages of uneven size in one
launch sequence, optionally replayed from a CUDA graph.

The batch must reproduce, bit for bit, what one dnni_interpolate_segment call
per tile gives (heights and site maps), whatever the order the tiles are
scheduled in, whether the sequence is captured in a graph, and whether the
tiles share input rows.  Points outside a tile's declared extent must fail
the run with DNNI_E_RANGE instead of being binned silently."""
import numpy as np
import pytest

from conftest import terrain_case

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def _tiles(seed=11, count=14):
    """Mixed tiles: sides 40-300 cells, cells 0.5/1/2 m, densities 0.05-4 per
    cell, own origins, some with halo rasters, plus edge cases (an empty tile,
    a one-point tile, a tile reusing another tile's rows)."""
    from terranni_b200 import engine
    rng = np.random.default_rng(seed)
    cases = []
    for k in range(count):
        side = int(np.exp(rng.uniform(np.log(40), np.log(300))))
        cell = int(rng.choice([50, 100, 200]))
        dens = float(np.exp(rng.uniform(np.log(0.05), np.log(4.0))))
        n = max(int(dens * side * side), 20)
        local = terrain_case(int(rng.integers(1, 1 << 30)), side, n, cell=cell, lakes=int(rng.integers(0, 4)),
                             lake_r=(0.05 * side, 0.3 * side))
        origin = (int(rng.integers(-5_000_000, 5_000_000)), int(rng.integers(-5_000_000, 5_000_000)))
        halo = int(rng.integers(0, 6)) if k % 3 == 0 else 0
        raster = (-halo, -halo, side + halo, side + halo) if halo else None
        wp = engine.make_wp(side, side, cell, origin[0], origin[1], raster=raster, z_offset=float(k))
        xyz = local.copy()
        xyz[:, 0] += origin[0]
        xyz[:, 1] += origin[1]
        cases.append({"wp": wp, "xyz": xyz})
    # a tile without points and a tile with one point
    cases.append({"wp": engine.make_wp(50, 37, 100, 1000, 2000), "xyz": np.zeros((0, 3), np.int32)})
    cases.append({"wp": engine.make_wp(33, 65, 100, -300, 700, raster=(-2, -2, 35, 67)),
                  "xyz": np.array([[-300 + 1234, 700 + 2345, 777]], np.int32)})
    return cases


def _layout(cases, share_rows=True, extent_pad=None):
    """Concatenated point rows, tile records and output offsets.  With
    share_rows the last real tile is added a second time on the same rows,
    under a coarser cell size."""
    from terranni_b200 import engine
    rows, tiles, meta = [], [], []
    pt = out = site = 0
    for k, c in enumerate(cases):
        wp, xyz = c["wp"], c["xyz"]
        x0, y0, x1, y1 = engine.raster_box(wp)
        ext = None
        if xyz.shape[0]:
            pad = extent_pad if extent_pad is not None else (0 if k % 2 else 5000)
            ext = (int(xyz[:, 0].min()) - pad, int(xyz[:, 1].min()) - pad,
                   int(xyz[:, 0].max()) + pad, int(xyz[:, 1].max()) + pad)
        tiles.append(engine.make_tile(wp, pt, xyz.shape[0], out, site, extent=ext))
        meta.append({"wp": wp, "pt": (pt, xyz.shape[0]), "out": out, "site": site, "sites": (y1 - y0, x1 - x0)})
        rows.append(xyz)
        pt += xyz.shape[0]
        out += wp.ncols * wp.nrows
        site += (y1 - y0) * (x1 - x0)
    if share_rows:
        k = len(cases) - 3
        c = cases[k]
        w0 = c["wp"]
        wp = engine.make_wp(w0.ncols // 2, w0.nrows // 2, w0.cell_size * 2, w0.origin_x, w0.origin_y)
        p0, n0 = meta[k]["pt"]
        t0 = tiles[k]
        tiles.append(engine.make_tile(wp, p0, n0, out, site, extent=(t0.ext_x0, t0.ext_y0, t0.ext_x1, t0.ext_y1)))
        meta.append({"wp": wp, "pt": (p0, n0), "out": out, "site": site, "sites": (wp.nrows, wp.ncols)})
        out += wp.ncols * wp.nrows
        site += wp.ncols * wp.nrows
    return np.concatenate(rows), tiles, meta, out, site


def _per_tile(eng, xyz, meta, gid=None):
    res = []
    for m in meta:
        p0, n = m["pt"]
        g = None if gid is None else gid[p0:p0 + n]
        h, s, _ = eng.interpolate(m["wp"], xyz[p0:p0 + n], g, site=True)
        res.append((h, s))
    return res


def _run_device(batch, xyz, nout, nsite, gid=None):
    import torch
    d_xyz = torch.from_numpy(xyz).cuda()
    d_gid = torch.from_numpy(gid.view(np.int32)).cuda() if gid is not None else None
    d_h = torch.full((max(nout, 1),), 7.0, dtype=torch.float32, device="cuda")
    d_s = torch.zeros((max(nsite, 1),), dtype=torch.int32, device="cuda")
    st = batch.run_device(d_xyz, d_h, d_gid=d_gid, d_site=d_s, stats=True)
    return d_h.cpu().numpy(), d_s.cpu().numpy().view(np.uint32), st


def _check(meta, ref, h, s):
    for m, (rh, rs) in zip(meta, ref):
        wp = m["wp"]
        got_h = h[m["out"]:m["out"] + wp.ncols * wp.nrows].reshape(wp.nrows, wp.ncols)
        got_s = s[m["site"]:m["site"] + rs.size].reshape(rs.shape)
        assert np.array_equal(got_s, rs)
        assert _same(got_h, rh)


@pytest.fixture(scope="module")
def eng():
    import torch
    from terranni_b200 import engine
    torch.cuda.set_device(0)
    e = engine.Engine(device=0)
    yield e
    e.close()


@pytest.mark.parametrize("use_graph,order_by_cost", [(False, False), (True, True)])
def test_batch_matches_per_tile_calls(eng, use_graph, order_by_cost):
    xyz, tiles, meta, nout, nsite = _layout(_tiles())
    ref = _per_tile(eng, xyz, meta)
    with eng.batch(tiles, use_graph=use_graph, order_by_cost=order_by_cost) as b:
        for _ in range(2):                     # second run replays the graph
            h, s, st = _run_device(b, xyz, nout, nsite)
            _check(meta, ref, h, s)
        assert st.n_cells == sum(m["wp"].ncols * m["wp"].nrows for m in meta)
        assert st.n_points == sum(m["pt"][1] for m in meta)


def test_batch_matches_oracle_on_small_tiles(eng, oracle):
    from terranni_b200 import engine
    cases = _tiles(seed=5, count=4)
    xyz, tiles, meta, nout, nsite = _layout(cases, share_rows=False)
    with eng.batch(tiles, use_graph=True) as b:
        h, s, _ = _run_device(b, xyz, nout, nsite)
    for m in meta:
        wp = m["wp"]
        p0, n = m["pt"]
        x0, y0, x1, y1 = engine.raster_box(wp)
        owp = oracle.make_wp(wp.ncols, wp.nrows, wp.cell_size, wp.origin_x, wp.origin_y, raster=(x0, y0, x1, y1),
                             z_offset=wp.z_offset)
        r = oracle.interpolate(owp, xyz[p0:p0 + n])
        assert np.array_equal(s[m["site"]:m["site"] + r["site"].size].reshape(r["site"].shape), r["site"])
        assert _same(h[m["out"]:m["out"] + wp.ncols * wp.nrows].reshape(wp.nrows, wp.ncols), r["h"])


def test_batch_with_gids_and_new_buffers(eng):
    xyz, tiles, meta, nout, nsite = _layout(_tiles(seed=3, count=8))
    gid = np.random.default_rng(1).permutation(xyz.shape[0]).astype(np.uint32)
    ref = _per_tile(eng, xyz, meta, gid)
    with eng.batch(tiles, use_graph=True, small_radius=2, bin_target=8) as b:
        for _ in range(2):                     # fresh buffers each run: the graph is re-captured
            h, s, _ = _run_device(b, xyz, nout, nsite, gid)
            _check(meta, ref, h, s)


def test_batch_host_path_matches_device_path(eng):
    xyz, tiles, meta, nout, nsite = _layout(_tiles(seed=9, count=6))
    with eng.batch(tiles) as b:
        h_d, s_d, _ = _run_device(b, xyz, nout, nsite)
        h = np.empty(nout, np.float32)
        s = np.empty(nsite, np.uint32)
        st = b.run(xyz, h, out_site=s)
    assert _same(h, h_d[:nout]) and np.array_equal(s, s_d[:nsite])
    assert st.h2d_bytes == xyz.nbytes and st.d2h_bytes == h.nbytes + s.nbytes


def test_batch_point_outside_declared_extent_is_a_range_error(eng):
    from terranni_b200 import engine
    xyz = terrain_case(4, 64, 3000)
    wp = engine.make_wp(64, 64, 100)
    tight = (0, 0, int(xyz[:, 0].max()) // 2, int(xyz[:, 1].max()))      # half the points lie outside
    with eng.batch([engine.make_tile(wp, 0, xyz.shape[0], 0, -1, extent=tight)]) as b:
        with pytest.raises(engine.DnniError) as ei:
            _run_device(b, xyz, 64 * 64, 0)
        assert ei.value.status == 5
        with pytest.raises(engine.DnniError) as ei:      # the host-buffer run checks without stats
            b.run(xyz, np.empty(64 * 64, np.float32), stats=False)
        assert ei.value.status == 5
    # a point beyond the bin grid of a tile planned from its raster alone
    far = np.concatenate([xyz, np.array([[900_000, 50, 10]], np.int32)])
    with eng.batch([engine.make_tile(wp, 0, far.shape[0], 0, -1)]) as b:
        with pytest.raises(engine.DnniError) as ei:
            _run_device(b, far, 64 * 64, 0)
        assert ei.value.status == 5
    with pytest.raises(engine.DnniError) as ei:          # extent beyond the coordinate range
        eng.batch([engine.make_tile(wp, 0, 10, 0, -1, extent=(0, 0, 1 << 30, 10))])
    assert ei.value.status == 5


def test_autotuned_options_give_the_same_heights(eng):
    import torch
    xyz, tiles, meta, nout, nsite = _layout(_tiles(seed=21, count=10))
    d_xyz = torch.from_numpy(xyz).cuda()
    opts, rep = eng.autotune(tiles, d_xyz, sample_tiles=6)
    assert rep["sample_tiles"] == 6 and len(rep["trials"]) >= 8
    assert rep["best"]["small_radius"] == opts["small_radius"] and rep["best"]["bin_target"] == opts["bin_target"]
    assert rep["best"]["ms"] <= rep["ms_default"] + 1e-6
    assert all(t["ms"] > 0 for t in rep["trials"])
    ref = _per_tile(eng, xyz, meta)
    with eng.batch(tiles, use_graph=True, **opts) as b:
        h, s, _ = _run_device(b, xyz, nout, nsite)
    _check(meta, ref, h, s)
    assert opts["dense_band"] in (16, 32, 64)
    assert {t["dense_band"] for t in rep["trials"]} == {16, 32, 64}


@pytest.mark.parametrize("dense_band,far_group", [(8, 2), (16, 1), (32, 2)])
def test_ring_search_block_shapes_give_the_same_result(eng, dense_band, far_group):
    """The ring search's pixel block (32 x dense_band pixels per staged bin
    window) is a tuning choice: every shape gives the per-tile result bit for
    bit, dense tiles included (a 200 x 200 tile at 8 points per cell, whose
    64-row windows do not fit in shared memory)."""
    from terranni_b200 import engine
    cases = _tiles(seed=31, count=8)
    dense = terrain_case(4242, 200, 320_000, lakes=2, lake_r=(10.0, 40.0))
    cases.insert(0, {"wp": engine.make_wp(200, 200, 100, raster=(-3, -3, 203, 203)), "xyz": dense})
    xyz, tiles, meta, nout, nsite = _layout(cases)
    ref = _per_tile(eng, xyz, meta)
    with eng.batch(tiles, use_graph=True, dense_band=dense_band, far_group=far_group) as b:
        h, s, _ = _run_device(b, xyz, nout, nsite)
    _check(meta, ref, h, s)


def test_bad_ring_search_block_shape_is_refused(eng):
    from terranni_b200 import engine
    xyz, tiles, meta, nout, nsite = _layout(_tiles(seed=5, count=2), share_rows=False)
    with pytest.raises(engine.DnniError):
        eng.batch(tiles, dense_band=24)


@pytest.mark.parametrize("reverse_out,ntiles", [(False, 20), (True, 20), (False, 6)])
def test_pipelined_host_run_matches_device_run(eng, reverse_out, ntiles):
    """Batches of 4 Mi point rows or more run their host-buffer form in
    slices whose upload, launches and download overlap (20 tiles: the full
    ramp of slices; 6 tiles: one tile per slice); the result must equal the
    device-buffer run, also when the tiles' outputs lie in the opposite order
    to their points."""
    from terranni_b200 import engine
    rng = np.random.default_rng(17)
    rows, tiles, sides = [], [], []
    pt = 0
    per = (4 << 20) // ntiles + 1   # point rows per tile: 4 Mi or more in all
    for k in range(ntiles):
        side = int(rng.integers(150, 400))
        n = int(rng.integers(per, per + 200_000))
        xyz = terrain_case(int(rng.integers(1, 1 << 30)), side, n, lakes=2, lake_r=(0.05 * side, 0.2 * side))
        xyz[:, 0] += 1_000_000 * k
        rows.append(xyz)
        sides.append(side)
        tiles.append((k, side, pt, n, xyz))
        pt += n
    xyz_all = np.concatenate(rows)
    assert xyz_all.shape[0] >= 4 << 20
    order = list(range(ntiles))[::-1] if reverse_out else list(range(ntiles))
    out = {}
    o = 0
    for k in order:
        out[k] = o
        o += sides[k] * sides[k]
    site = {}
    sp = 0
    for k in range(ntiles):
        site[k] = sp
        sp += sides[k] * sides[k]
    tl = []
    for k, side, p0, n, xyz in tiles:
        wp = engine.make_wp(side, side, 100, 1_000_000 * k, 0)
        ext = (int(xyz[:, 0].min()), int(xyz[:, 1].min()), int(xyz[:, 0].max()), int(xyz[:, 1].max()))
        tl.append(engine.make_tile(wp, p0, n, out[k], site[k], extent=ext))
    gid = rng.permutation(xyz_all.shape[0]).astype(np.uint32)
    with eng.batch(tl, use_graph=True) as b:
        h_d, s_d, _ = _run_device(b, xyz_all, o, sp, gid)
        h = np.empty(o, np.float32)
        s = np.empty(sp, np.uint32)
        for _ in range(2):
            st = b.run(xyz_all, h, gid=gid, out_site=s)
            assert _same(h, h_d[:o]) and np.array_equal(s, s_d[:sp])
        assert st.n_cells == o and st.ms_total > 0
