"""The reference's default semantics on the GPU (dnni_interpolate_compat):
square site and query regions on a finer pixel lattice, float32 plane
depths with the later-drawn site winning ties, int32 z-codes with a
truncating divide.  The kernels must reproduce the oracle's restatement of
those rules (oracle.compat) exactly: the int32 division results and the
float32 heights bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    from terranni_b200 import engine
    e = engine.Engine(device=0)
    yield e
    e.close()


def _cases():
    rng = np.random.default_rng(21)
    out = []
    # terranni's CLI defaults: scaling 5, cell 2 m, site radius 5 m, query radius blockWidth*cell/2 - 0.01
    pts = np.stack([rng.uniform(0, 80, 3000), rng.uniform(0, 60, 3000), rng.uniform(10, 20, 3000)], 1)
    out.append(dict(scale=5, cell=2.0, sr=5.0, qr=4.99, pmin=0, ncols=40, nrows=30, origin=(0.0, 0.0), pts=pts))
    # one-to-one lattice, an origin, repeated positions (the later draw wins equal depths), sparse corners
    xy = np.stack([rng.uniform(1000, 1064, 900), rng.uniform(2000, 2048, 900)], 1)
    xy = np.concatenate([xy, xy[:200]])
    z = rng.uniform(-5, 40, xy.shape[0])
    out.append(dict(scale=1, cell=1.0, sr=3.0, qr=2.5, pmin=-6, ncols=64, nrows=48, origin=(1000.0, 2000.0),
                    pts=np.concatenate([xy, z[:, None]], 1)))
    # scaling 2, wide site squares, few points
    pts = np.stack([rng.uniform(0, 30, 120), rng.uniform(0, 30, 120), rng.uniform(100, 130, 120)], 1)
    out.append(dict(scale=2, cell=1.5, sr=8.0, qr=6.0, pmin=99, ncols=20, nrows=20, origin=(0.0, 0.0), pts=pts))
    # UTM-scale world coordinates: the float32 work-package origin and the
    # double points meet in the subtraction, as in the reference
    pts = np.stack([rng.uniform(500100, 500180, 2500), rng.uniform(4100200, 4100260, 2500),
                    rng.uniform(200, 230, 2500)], 1)
    out.append(dict(scale=5, cell=2.0, sr=5.0, qr=4.99, pmin=150, ncols=40, nrows=30, origin=(500100.0, 4100200.0),
                    pts=pts))
    return out


@pytest.mark.parametrize("k", range(4))
def test_compat_matches_oracle(eng, oracle, k):
    from terranni_b200 import engine
    c = _cases()[k]
    zmax = float(c["pts"][:, 2].max())
    mult = oracle.compat_multiplier(c["sr"], c["scale"], c["cell"], zmax, c["pmin"])
    so = oracle.CompatSettings(scale=c["scale"], cell_size=c["cell"], site_radius=c["sr"], query_radius=c["qr"],
                               point_min=c["pmin"], multiplier=mult, total_ncols=c["ncols"], total_nrows=c["nrows"])
    wo = oracle.CompatWP(origin_x=c["origin"][0], origin_y=c["origin"][1], grid_origin_x=0.0, grid_origin_y=0.0,
                         nrows=c["nrows"], ncols=c["ncols"])
    ref_h, ref_res = oracle.compat(so, wo, c["pts"])
    se = engine.CompatSettings(scale=c["scale"], cell_size=c["cell"], site_radius=c["sr"], query_radius=c["qr"],
                               point_min=c["pmin"], multiplier=mult, total_ncols=c["ncols"], total_nrows=c["nrows"])
    we = engine.CompatWP(origin_x=c["origin"][0], origin_y=c["origin"][1], grid_origin_x=0.0, grid_origin_y=0.0,
                         nrows=c["nrows"], ncols=c["ncols"])
    h, res = eng.interpolate_compat(se, we, c["pts"])
    assert np.array_equal(res, ref_res)
    assert np.array_equal(h.view(np.uint32), ref_h.view(np.uint32))
    assert (ref_h != np.float32(-9999.0)).mean() > 0.5


def test_compat_rejects_bad_settings(eng):
    from terranni_b200 import engine
    se = engine.CompatSettings(scale=0, cell_size=1.0, site_radius=1.0, query_radius=1.0, point_min=0, multiplier=1)
    we = engine.CompatWP(nrows=4, ncols=4)
    with pytest.raises(engine.DnniError) as ei:
        eng.interpolate_compat(se, we, np.zeros((1, 3)))
    assert ei.value.status == 1


def test_compat_device_buffers_equal_host_buffers(eng, oracle):
    import torch
    from terranni_b200 import engine
    c = _cases()[0]
    zmax = float(c["pts"][:, 2].max())
    mult = oracle.compat_multiplier(c["sr"], c["scale"], c["cell"], zmax, c["pmin"])
    se = engine.CompatSettings(scale=c["scale"], cell_size=c["cell"], site_radius=c["sr"], query_radius=c["qr"],
                               point_min=c["pmin"], multiplier=mult, total_ncols=c["ncols"], total_nrows=c["nrows"])
    we = engine.CompatWP(origin_x=c["origin"][0], origin_y=c["origin"][1], grid_origin_x=0.0, grid_origin_y=0.0,
                         nrows=c["nrows"], ncols=c["ncols"])
    h, res = eng.interpolate_compat(se, we, c["pts"])
    d_pts = torch.from_numpy(np.ascontiguousarray(c["pts"], np.float64)).cuda()
    d_h = torch.zeros(c["nrows"] * c["ncols"], dtype=torch.float32, device="cuda")
    d_r = torch.zeros(c["nrows"] * c["ncols"], dtype=torch.int32, device="cuda")
    eng.interpolate_compat_device(se, we, d_pts, c["pts"].shape[0], d_h, d_r,
                                  stream=torch.cuda.current_stream().cuda_stream)
    assert np.array_equal(d_h.cpu().numpy().reshape(h.shape).view(np.uint32), h.view(np.uint32))
    assert np.array_equal(d_r.cpu().numpy().reshape(res.shape), res)
