"""dnni_measure_peaks: the device's measured throughput of the operations
that bound the hot path's kernels (the denominators of their op-count
rooflines) is positive and of the order a B200 sustains."""
import pytest

pytestmark = pytest.mark.gpu


def test_measured_peaks_are_plausible():
    from terranni_b200 import engine
    p = engine.measure_peaks(0)
    assert p["sm_count"] > 0 and p["sm_clock_mhz"] > 0
    assert p["int_ops_per_s"] > 1e12          # integer multiply-adds, all SMs
    assert p["smem_atomics_per_s"] > 1e11     # shared-memory atomic adds
    assert p["l2_red64_per_s"] > 1e10         # L2 64-bit reductions


def test_batch_statistics_split_the_nearest_phase():
    import numpy as np
    import torch
    from conftest import terrain_case
    from terranni_b200 import engine
    xyz = terrain_case(3, 300, 30000, lakes=3, lake_r=(20.0, 60.0))
    tiles = [engine.make_tile(engine.make_wp(300, 300, 100), 0, xyz.shape[0], 0)]
    with engine.Engine(device=0) as e, e.batch(tiles) as b:
        d_xyz = torch.from_numpy(np.ascontiguousarray(xyz)).cuda()
        d_h = torch.empty(300 * 300, dtype=torch.float32, device="cuda")
        st = b.run_device(d_xyz, d_h, stats=True)
    assert 0 < st.ms_dense <= st.ms_nearest + 1e-6 and st.ms_far >= 0
    assert st.evals_dense > 0 and st.evals_far > 0
    assert sum(st.span_hist) == st.spans
