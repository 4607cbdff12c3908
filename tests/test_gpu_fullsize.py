"""The single-tile workload at its full size: a 4096 x 4096 grid at 1 m from
20 M points (70 % uniform, 30 % in 64 Gaussian clusters, 16 empty lakes of
radius 50-400 m, fBm terrain), one work package through the C ABI, checked
against the oracle's restatement of nni::performNNI (nni.cpp:870-944): the
site map and the float32 heights bit for bit, and every height within
1e-4 m of the FP64 value of its exact integer sums."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL_M = 1e-4


def test_tile4096_full_size_against_the_oracle(oracle):
    from terranni_b200 import engine, synth
    w = synth.config2()
    side = w["ncols"]
    wp = engine.make_wp(side, side, 100)
    with engine.Engine(device=0) as e:
        h, site, st = e.interpolate(wp, w["xyz"], site=True)
    ref = oracle.interpolate(oracle.make_wp(side, side, 100), w["xyz"])
    assert np.array_equal(site, ref["site"])
    assert np.array_equal(h.view(np.uint32), ref["h"].view(np.uint32))
    ok = ref["C"] > 0
    truth = oracle.exact_height_f64(ref["Z"][ok], ref["C"][ok], wp.z_scale, wp.z_offset)
    err = np.abs(h[ok].astype(np.float64) - truth)
    assert err.max() <= TOL_M and np.sqrt(np.mean(err * err)) <= TOL_M
    # lakes make discs of hundreds of cells: the span path and the far pass
    # both carry real work here
    assert st.max_r2 > 100 ** 2 and st.big_pixels > 0 and st.nodata_cells == 0
