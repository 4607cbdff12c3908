"""Serving (dnni_server_*): DEM requests against a resident cloud, with
continuous batching.

A request's result is defined without reference to batching: the window of
the interpolation whose raster is the cloud's bounding box on the request's
cell lattice, every point of the cloud a site.  The tests check that
definition directly (one work package with that whole raster), that each
result is bit-identical alone and in a mix submitted from several threads at
once, and that admission by device footprint rejects what cannot fit."""
import threading

import numpy as np
import pytest

from conftest import terrain_case

pytestmark = pytest.mark.gpu
SIDE, CELL = 1200, 100          # world: 1200 x 1200 cells of 1 m = 120000 LAS units


@pytest.fixture(scope="module")
def eng():
    import torch
    from terranni_b200 import engine
    torch.cuda.set_device(0)
    e = engine.Engine(device=0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def cloud():
    xyz = terrain_case(77, SIDE, 300_000, lakes=4, lake_r=(20.0, 120.0))
    return xyz + np.array([3_000_000, 7_000_000, 0], np.int32)


def _requests(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        cs = int(rng.choice([50, 100, 200]))
        side_m = float(np.exp(rng.uniform(np.log(20.0), np.log(500.0))))
        n = max(4, int(side_m * 100 / cs))
        m = max(4, int(n * rng.uniform(0.6, 1.4)))
        x0 = 3_000_000 + int(rng.integers(-20_000, 120_000))
        y0 = 7_000_000 + int(rng.integers(-20_000, 120_000))
        out.append(dict(x0=x0, y0=y0, ncols=n, nrows=m, cell_size=cs, site=bool(k % 2)))
    out.append(dict(x0=3_000_000 - 500_000, y0=7_000_000, ncols=30, nrows=20, cell_size=100, site=True))  # off the cloud
    return out


def _world_wp(engine, xyz, r):
    """One work package: the request's grid, raster = the cloud's box on its lattice."""
    cs = r["cell_size"]
    wx0, wy0 = int(xyz[:, 0].min()), int(xyz[:, 1].min())
    wx1, wy1 = int(xyz[:, 0].max()), int(xyz[:, 1].max())
    i0 = -((r["x0"] - wx0) // cs)
    i1 = (wx1 - r["x0"]) // cs
    j0 = -((r["y0"] - wy0) // cs)
    j1 = (wy1 - r["y0"]) // cs
    return engine.make_wp(r["ncols"], r["nrows"], cs, r["x0"], r["y0"], raster=(i0, j0, i1 + 1, j1 + 1)), (i0, j0)


def test_server_results_match_the_definition_and_the_mix(eng, cloud):
    from terranni_b200 import engine
    reqs = _requests(5, 14)
    with eng.server(cloud, slots=2, max_batch=4, slot_bytes=512 << 20) as srv:
        alone = []
        for r in reqs:
            t = srv.submit(**r)
            alone.append(srv.wait(t, timeout=120))
        # the mix: all requests at once from three threads
        tickets = [None] * len(reqs)

        def client(ks):
            for k in ks:
                tickets[k] = srv.submit(**reqs[k])
        th = [threading.Thread(target=client, args=(list(range(i, len(reqs), 3)),)) for i in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        mix = [srv.wait(t, timeout=120) for t in tickets]
        st = srv.stats()
    assert st["completed"] == 2 * len(reqs) and st["failed"] == 0
    assert max(m[2]["batch_size"] for m in mix) > 1
    # the slots' device time line: busy time, overlap of two slots within it
    assert st["ms_device_busy"] > 0 and 0 <= st["ms_device_overlap"] <= st["ms_device_busy"] + 1e-6
    assert st["ms_device_span"] >= st["ms_device_busy"] - 1e-6
    for (ha, sa, ra), (hm, smx, rm) in zip(alone, mix):
        assert np.array_equal(ha.view(np.uint32), hm.view(np.uint32))
        if sa is not None:
            assert np.array_equal(sa, smx)
    # the definition, on the requests inside the cloud's box
    for r, (h, s, res) in list(zip(reqs, alone))[:6]:
        wp, (i0, j0) = _world_wp(engine, cloud, r)
        rh, rs, _ = eng.interpolate(wp, cloud, site=True)
        assert np.array_equal(h.view(np.uint32), rh.view(np.uint32))
        if s is not None:
            ys, xs = np.mgrid[0:r["nrows"], 0:r["ncols"]]
            inside = (xs >= i0) & (ys >= j0) & (xs - i0 < rs.shape[1]) & (ys - j0 < rs.shape[0])
            assert np.array_equal(s[inside], rs[(ys - j0)[inside], (xs - i0)[inside]])
            assert np.all(s[~inside] == 0xFFFFFFFF)
    off = alone[-1]
    assert np.all(off[0] == np.float32(-9999.0)) and np.all(off[1] == 0xFFFFFFFF)


def test_server_results_against_the_oracle(eng, cloud, oracle):
    # served windows checked directly against the oracle's interpolation of
    # the definition (the request's grid, raster = the cloud's box on its
    # lattice): heights and site map bit for bit, FP64 error within 1e-4 m
    from terranni_b200 import engine
    reqs = [dict(x0=3_020_000, y0=7_015_000, ncols=180, nrows=140, cell_size=100, site=True),
            dict(x0=3_055_500, y0=7_060_700, ncols=90, nrows=120, cell_size=200, site=True)]
    with eng.server(cloud, slots=2, max_batch=4, slot_bytes=512 << 20) as srv:
        tickets = [srv.submit(**r) for r in reqs]
        got = [srv.wait(t, timeout=120) for t in tickets]
    for r, (h, s, _) in zip(reqs, got):
        wp, (i0, j0) = _world_wp(engine, cloud, r)
        owp = oracle.make_wp(r["ncols"], r["nrows"], r["cell_size"], r["x0"], r["y0"],
                             raster=(wp.raster_x0, wp.raster_y0, wp.raster_x1, wp.raster_y1))
        ref = oracle.interpolate(owp, cloud)
        assert np.array_equal(h.view(np.uint32), ref["h"].view(np.uint32))
        ys, xs = np.mgrid[0:r["nrows"], 0:r["ncols"]]
        assert np.array_equal(s, ref["site"][ys - j0, xs - i0])
        ok = ref["C"] > 0
        truth = oracle.exact_height_f64(ref["Z"][ok], ref["C"][ok], 0.01, 0.0)
        assert np.abs(h[ok].astype(np.float64) - truth).max() <= 1e-4


def test_server_rejects_a_request_beyond_its_slot(eng, cloud):
    from terranni_b200 import engine
    with eng.server(cloud, slots=1, slot_bytes=64 << 20) as srv:
        t = srv.submit(3_000_000, 7_000_000, 6000, 6000, 20)       # ~36 M cells: beyond 64 MiB
        with pytest.raises(engine.DnniError) as ei:
            srv.wait(t, timeout=60)
        assert ei.value.status == 2
        t = srv.submit(3_000_000, 7_000_000, 64, 64, 100)
        h, _, res = srv.wait(t, timeout=60)
        assert res["status"] == 0 and h.shape == (64, 64)
