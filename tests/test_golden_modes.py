"""Known answers for the reference-default and space-time modes
(tests/golden/golden_modes.npz, from make_golden_modes.py): the oracle on the
CPU, and the engine on the GPU through the C ABI, both bit for bit."""
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G = np.load(os.path.join(ROOT, "tests", "golden", "golden_modes.npz"))
NC, NS = int(G["n_compat"][0]), int(G["n_st"][0])


def _compat_args(mod, k):
    p = G[f"compat{k}_params"]
    scale, cell, sr, qr, pmin, mult, ox, oy, nrows, ncols = p
    s = mod.CompatSettings(scale=int(scale), cell_size=float(cell), site_radius=float(sr), query_radius=float(qr),
                           point_min=int(pmin), multiplier=int(mult), total_ncols=int(ncols), total_nrows=int(nrows))
    wp = mod.CompatWP(origin_x=float(ox), origin_y=float(oy), grid_origin_x=0.0, grid_origin_y=0.0,
                      nrows=int(nrows), ncols=int(ncols))
    return s, wp, G[f"compat{k}_pts"]


def _st_args(mod, k):
    ncols, nrows, cs, rx0, ry0, rx1, ry1, cur, rt, tau = (int(v) for v in G[f"st{k}_params"])
    return mod.make_wp(ncols, nrows, cs, raster=(rx0, ry0, rx1, ry1)), G[f"st{k}_xyz"], G[f"st{k}_t"], cur, rt, tau


@pytest.mark.parametrize("k", range(NC))
def test_oracle_compat_golden(oracle, k):
    s, wp, pts = _compat_args(oracle, k)
    h, res = oracle.compat(s, wp, pts)
    assert np.array_equal(res, G[f"compat{k}_res"])
    assert np.array_equal(h.view(np.uint32), G[f"compat{k}_h"].view(np.uint32))


@pytest.mark.parametrize("k", range(NS))
def test_oracle_spacetime_golden(oracle, k):
    wp, xyz, t, cur, rt, tau = _st_args(oracle, k)
    r = oracle.interpolate_spacetime(wp, xyz, t, cur, rt, tau)
    assert np.array_equal(r["Z"], G[f"st{k}_Z"]) and np.array_equal(r["C"], G[f"st{k}_C"])
    assert np.array_equal(r["h"].view(np.uint32), G[f"st{k}_h"].view(np.uint32))


@pytest.fixture(scope="module")
def eng():
    from terranni_b200 import engine
    e = engine.Engine(device=0)
    yield e
    e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(NC))
def test_engine_compat_golden(eng, k):
    from terranni_b200 import engine
    s, wp, pts = _compat_args(engine, k)
    h, res = eng.interpolate_compat(s, wp, pts)
    assert np.array_equal(res, G[f"compat{k}_res"])
    assert np.array_equal(h.view(np.uint32), G[f"compat{k}_h"].view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(NS))
def test_engine_spacetime_golden(eng, k):
    from terranni_b200 import engine
    wp, xyz, t, cur, rt, tau = _st_args(engine, k)
    h, _ = eng.interpolate_spacetime(wp, xyz, t, cur, rt, tau)
    assert np.array_equal(h.view(np.uint32), G[f"st{k}_h"].view(np.uint32))
