"""Geometry at the engine's limits, bit-exact against the oracle: grid sides
of 32767 cells (the largest a work package takes), coordinates reaching
towards +-2^30 LAS units from the origin, and such a strip inside a batch
beside an ordinary tile (index arithmetic that overflows 32 bits, or a
stride mixed up between rows and columns, shows here first)."""
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


def _strip(seed, ncols, nrows, cs, n, ox=0, oy=0):
    rng = np.random.default_rng(seed)
    xyz = np.stack([rng.integers(0, ncols * cs, n) + ox, rng.integers(0, nrows * cs, n) + oy,
                    rng.integers(-20000, 90000, n)], 1).astype(np.int32)
    return xyz


@pytest.mark.parametrize("ncols,nrows", [(32767, 40), (40, 32767)])
def test_longest_side(eng, oracle, ncols, nrows):
    from terranni_b200 import engine
    xyz = _strip(3, ncols, nrows, 100, 150_000)
    ref = oracle.interpolate(oracle.make_wp(ncols, nrows, 100), xyz)
    h, site, _ = eng.interpolate(engine.make_wp(ncols, nrows, 100), xyz, site=True)
    assert np.array_equal(site, ref["site"]) and _same(h, ref["h"])


def test_coordinates_towards_the_range_limit(eng, oracle):
    # 2000 x 40 cells of 500 000 LAS units: the grid spans 10^9 units (2^30 is
    # 1.07 * 10^9), with the origin far from zero and a raster halo
    from terranni_b200 import engine
    cs = 500_000
    ox, oy = -2_000_000_000, 1_500_000_000
    xyz = _strip(5, 2000, 40, cs, 60_000, ox, oy)
    xyz[:, 0] = np.clip(xyz[:, 0].astype(np.int64), ox, ox + 1999 * cs).astype(np.int32)
    args = dict(origin_x=ox, origin_y=oy, raster=(-1, -1, 2001, 41))
    ref = oracle.interpolate(oracle.make_wp(2000, 40, cs, **args), xyz)
    h, site, _ = eng.interpolate(engine.make_wp(2000, 40, cs, **args), xyz, site=True)
    assert np.array_equal(site, ref["site"]) and _same(h, ref["h"])
    assert (ref["h"] != np.float32(-9999.0)).all()


def test_longest_side_in_a_batch(eng, oracle):
    import torch
    from terranni_b200 import engine
    a = _strip(7, 32767, 32, 100, 120_000)
    b = _strip(8, 300, 200, 50, 40_000, 7_000_000, -3_000_000)
    xyz = np.concatenate([a, b])
    wa = engine.make_wp(32767, 32, 100)
    wb = engine.make_wp(300, 200, 50, 7_000_000, -3_000_000, raster=(-2, -2, 302, 202))
    na, nb = 32767 * 32, 300 * 200
    ext = lambda p: (int(p[:, 0].min()), int(p[:, 1].min()), int(p[:, 0].max()), int(p[:, 1].max()))
    tiles = [engine.make_tile(wa, 0, a.shape[0], 0, 0, extent=ext(a)),
             engine.make_tile(wb, a.shape[0], b.shape[0], na, na, extent=ext(b))]
    with eng.batch(tiles, use_graph=True) as bt:
        d_xyz = torch.from_numpy(xyz).cuda()
        d_h = torch.zeros(na + nb, dtype=torch.float32, device="cuda")
        d_s = torch.zeros(na + 304 * 204, dtype=torch.int32, device="cuda")
        # queued on torch's stream, so that the copies below follow it
        bt.run_device(d_xyz, d_h, d_site=d_s, stream=torch.cuda.current_stream().cuda_stream)
        h = d_h.cpu().numpy()
        s = d_s.cpu().numpy().view(np.uint32)
    ra = oracle.interpolate(oracle.make_wp(32767, 32, 100), a)
    rb = oracle.interpolate(oracle.make_wp(300, 200, 50, 7_000_000, -3_000_000, raster=(-2, -2, 302, 202)), b)
    assert _same(h[:na].reshape(32, 32767), ra["h"]) and np.array_equal(s[:na].reshape(32, 32767), ra["site"])
    assert _same(h[na:].reshape(200, 300), rb["h"]) and np.array_equal(s[na:].reshape(204, 304), rb["site"])
