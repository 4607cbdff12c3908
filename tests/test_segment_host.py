"""Host-side parts of the segment driver, on the CPU: the exact squared
distance transform that bounds each tile's halo, against brute force."""
import ctypes

import numpy as np
import pytest


def _edt(emu_lib, occ):
    ny, nx = occ.shape
    out = np.empty((ny, nx), np.float64)
    emu_lib.emu_edt_2d.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    emu_lib.emu_edt_2d.restype = None
    o = np.ascontiguousarray(occ, np.uint8)
    emu_lib.emu_edt_2d(o.ctypes.data, nx, ny, out.ctypes.data)
    return out


@pytest.fixture(scope="module")
def emu_lib(emu):
    from conftest import EMU_SO
    return ctypes.CDLL(EMU_SO)


@pytest.mark.parametrize("seed,nx,ny,frac", [(1, 37, 23, 0.05), (2, 64, 64, 0.002), (3, 1, 40, 0.1),
                                             (4, 50, 1, 0.1), (5, 30, 30, 0.9)])
def test_edt_matches_brute_force(emu_lib, seed, nx, ny, frac):
    rng = np.random.default_rng(seed)
    occ = (rng.random((ny, nx)) < frac).astype(np.uint8)
    occ[rng.integers(0, ny), rng.integers(0, nx)] = 1
    got = _edt(emu_lib, occ)
    ys, xs = np.nonzero(occ)
    gy, gx = np.mgrid[0:ny, 0:nx]
    want = ((gx[..., None] - xs) ** 2 + (gy[..., None] - ys) ** 2).min(axis=-1)
    assert np.array_equal(got, want.astype(np.float64))


def test_edt_of_an_empty_grid_is_far(emu_lib):
    got = _edt(emu_lib, np.zeros((5, 7), np.uint8))
    assert np.all(got >= 1e19)
