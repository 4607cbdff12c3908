"""The C++ drop-in for TerraNNI's nni:: interface (include/nni/nni.h).

A caller written against the reference's interface, the way binRun
(terranni.cpp:394-426) drives it, is compiled against the shim and linked
with libdnni.so (CPU test); on a GPU its OutPoint stream must equal the
oracle's heights for the same work package, in the reference's order
(nni.cpp:836-858: i-major, clipped to the global grid)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "nni_shim_demo.cpp")
EXE = os.path.join(ROOT, "tests", "native", "nni_shim_demo")
LIBDIR = os.path.join(ROOT, "terranni_b200")

POINT4D = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("t", "<i4"), ("pad", "<i4")])
OUTPOINT = np.dtype([("i", "<i4"), ("j", "<i4"), ("h", "<f4")])


TSRC = os.path.join(ROOT, "tests", "native", "nni_shim_time_demo.cpp")
TEXE = os.path.join(ROOT, "tests", "native", "nni_shim_time_demo")


def build_demo(src=SRC, exe=EXE):
    deps = [src, os.path.join(ROOT, "include", "nni", "nni.h"), os.path.join(ROOT, "include", "tpie", "stream.h"),
            os.path.join(ROOT, "include", "dnni.h"), os.path.join(LIBDIR, "libdnni.so")]
    if not os.path.exists(exe) or any(os.path.getmtime(d) > os.path.getmtime(exe) for d in deps):
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), src, "-o", exe,
               "-L", LIBDIR, "-ldnni", f"-Wl,-rpath,{LIBDIR}"]
        subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_reference_caller_compiles_and_links_against_the_shim():
    exe = build_demo()
    assert os.access(exe, os.X_OK)
    assert os.access(build_demo(TSRC, TEXE), os.X_OK)
    assert POINT4D.itemsize == 32 and OUTPOINT.itemsize == 12     # nni.h:34-64 layouts


@pytest.mark.gpu
def test_reference_caller_matches_oracle(tmp_path, oracle):
    from conftest import terrain_case
    exe = build_demo()
    ncols, nrows, cell_m, qr = 90, 70, 1.0, 3.0
    ox, oy = 1000.0, 2000.0                      # exactly representable as float
    gox, goy, tot_c, tot_r = 10, 20, 95, 85      # the work package's last 5 columns fall outside
    xyz = terrain_case(17, 100, 6000, lakes=1, lake_r=(5.0, 15.0))
    xyz = xyz - np.array([500, 500, 0], np.int32)           # some points in the halo, some negative
    pts = np.zeros(xyz.shape[0], POINT4D)
    pts["x"] = ox + xyz[:, 0] * 0.01
    pts["y"] = oy + xyz[:, 1] * 0.01
    pts["z"] = xyz[:, 2] * 0.01
    pin, pout = tmp_path / "pts.bin", tmp_path / "out.bin"
    pts.tofile(pin)
    r = subprocess.run([exe, str(pin), str(pout), str(ncols), str(nrows), str(cell_m), str(ox), str(oy), str(gox),
                        str(goy), str(tot_c), str(tot_r), str(qr)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(pout, OUTPOINT)
    po = int(np.ceil(qr / cell_m)) + 1           # nni.cpp:881-883 with scale 1
    wp = oracle.make_wp(ncols, nrows, 100, raster=(-po, -po, ncols + po, nrows + po))
    ref = oracle.interpolate(wp, xyz)["h"]
    want = [(i + gox, j + goy, ref[j, i]) for i in range(ncols) for j in range(nrows)
            if i + gox < tot_c and j + goy < tot_r]
    assert got.shape[0] == len(want)
    assert np.array_equal(got["i"], np.array([w[0] for w in want], np.int32))
    assert np.array_equal(got["j"], np.array([w[1] for w in want], np.int32))
    assert np.array_equal(got["h"].view(np.uint32), np.array([w[2] for w in want], np.float32).view(np.uint32))


@pytest.mark.gpu
def test_reference_caller_compat_mode_matches_oracle(tmp_path, oracle):
    """nni::setCompatMode: the same caller, the reference's default semantics
    (scaling 5, site radius 5 m, pointMin/multiplier quantisation)."""
    exe = build_demo()
    ncols, nrows, cell_m, qr, scale, sr, pmin = 40, 30, 2.0, 4.99, 5, 5.0, 0
    ox, oy, gox, goy, tot_c, tot_r = 500.0, 700.0, 3, 4, 40, 32
    rng = np.random.default_rng(9)
    n = 3000
    pts = np.zeros(n, POINT4D)
    pts["x"] = ox + rng.uniform(-4, 84, n)
    pts["y"] = oy + rng.uniform(-4, 64, n)
    pts["z"] = rng.uniform(10, 20, n)
    mult = oracle.compat_multiplier(sr, scale, cell_m, float(pts["z"].max()), pmin)
    pin, pout = tmp_path / "pts.bin", tmp_path / "out.bin"
    pts.tofile(pin)
    r = subprocess.run([exe, str(pin), str(pout), str(ncols), str(nrows), str(cell_m), str(ox), str(oy), str(gox),
                        str(goy), str(tot_c), str(tot_r), str(qr), str(scale), str(sr), str(pmin), str(mult)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(pout, OUTPOINT)
    s = oracle.CompatSettings(scale=scale, cell_size=cell_m, site_radius=sr, query_radius=qr, point_min=pmin,
                              multiplier=mult, total_ncols=tot_c, total_nrows=tot_r)
    cwp = oracle.CompatWP(origin_x=ox, origin_y=oy, grid_origin_x=gox, grid_origin_y=goy, nrows=nrows, ncols=ncols)
    ref, _ = oracle.compat(s, cwp, np.stack([pts["x"], pts["y"], pts["z"]], 1))
    want = [(i + gox, j + goy, ref[j, i]) for i in range(ncols) for j in range(nrows)
            if i + gox < tot_c and j + goy < tot_r]
    assert got.shape[0] == len(want)
    assert np.array_equal(got["i"], np.array([w[0] for w in want], np.int32))
    assert np.array_equal(got["h"].view(np.uint32), np.array([w[2] for w in want], np.float32).view(np.uint32))
    assert (ref != np.float32(-9999.0)).mean() > 0.9


@pytest.mark.gpu
@pytest.mark.parametrize("rt,delta", [(1, 1), (1, 0), (2, 1), (2, 0)])
def test_space_time_caller_matches_oracle(tmp_path, oracle, rt, delta):
    """binRun's time loop (terranni.cpp:408-420) over one work package: every
    curTime's OutPoints equal the oracle's space-time interpolation of the
    whole time-sorted stream, and the stream is left where the reference's
    seeks leave it (Delta: the first point of time cur + 1; Delta^2: of time
    cur + 1 - 2 rt, nni.cpp:782-788)."""
    from conftest import terrain_case
    exe = build_demo(TSRC, TEXE)
    side, cell_m, qr, t0, t1 = 60, 1.0, 3.0, 3, 7
    xyz = terrain_case(23, side, 5000, lakes=1, lake_r=(5.0, 15.0))
    times = np.sort(np.random.default_rng(4).integers(0, 11, xyz.shape[0])).astype(np.int32)
    pts = np.zeros(xyz.shape[0], POINT4D)
    pts["x"], pts["y"], pts["z"], pts["t"] = xyz[:, 0] * 0.01, xyz[:, 1] * 0.01, xyz[:, 2] * 0.01, times
    pin = tmp_path / "pts.bin"
    pts.tofile(pin)
    r = subprocess.run([exe, str(pin), str(tmp_path / "out_"), str(side), str(side), str(cell_m), str(qr), str(rt),
                        str(t0), str(t1), str(delta)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    pos = {int(a[1]): int(a[3]) for a in (ln.split() for ln in r.stdout.splitlines()) if a[0] == "t"}
    po = int(np.ceil(qr / cell_m)) + 1
    wp = oracle.make_wp(side, side, 100, raster=(-po, -po, side + po, side + po))
    for cur in range(t0, t1 + 1):
        got = np.fromfile(tmp_path / f"out_{cur}.bin", OUTPOINT)
        ref = oracle.interpolate_spacetime(wp, xyz, times, cur, rt, 100)["h"]
        want = np.array([ref[j, i] for i in range(side) for j in range(side)], np.float32)
        assert np.array_equal(got["h"].view(np.uint32), want.view(np.uint32))
        first = cur + 1 if delta else cur + 1 - 2 * rt
        assert pos[cur] == int(np.searchsorted(times, first))


def _stub_build(tmp_path):
    """The time demo linked against tests/native/dnni_stub.c (no GPU)."""
    lib = tmp_path / "libdnni.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-std=c99", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "native", "dnni_stub.c"), "-o", str(lib)], check=True,
                   capture_output=True, text=True)
    exe = tmp_path / "time_demo"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), TSRC, "-o", str(exe),
                    "-L", str(tmp_path), "-ldnni", f"-Wl,-rpath,{tmp_path}"], check=True, capture_output=True,
                   text=True)
    return exe


@pytest.mark.parametrize("rt,delta", [(1, 1), (1, 0), (2, 1), (2, 0)])
def test_space_time_stream_handling_on_cpu(tmp_path, rt, delta):
    """The drop-in's space-time reads (nni.cpp:750-788), seeks and Delta-mode
    slice reuse (nni.cpp:325-359), with a stub engine: each call hands the
    engine exactly the points within 2 rt of its time, and the stream ends
    where the reference's seeks leave it."""
    exe = _stub_build(tmp_path)
    rng = np.random.default_rng(3)
    n = 4000
    times = np.sort(rng.integers(0, 13, n)).astype(np.int32)
    pts = np.zeros(n, POINT4D)
    pts["x"], pts["y"], pts["z"], pts["t"] = rng.uniform(0, 30, n), rng.uniform(0, 30, n), 1.0, times
    pin = tmp_path / "pts.bin"
    pts.tofile(pin)
    log = tmp_path / "calls.log"
    t0, t1 = 4, 8
    env = dict(os.environ, DNNI_STUB_LOG=str(log))
    r = subprocess.run([str(exe), str(pin), str(tmp_path / "out_"), "30", "30", "1.0", "3.0", str(rt), str(t0),
                        str(t1), str(delta)], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    pos = {int(a[1]): int(a[3]) for a in (ln.split() for ln in r.stdout.splitlines()) if a[0] == "t"}
    calls = [ln.split() for ln in log.read_text().splitlines()]
    assert [c[0] for c in calls] == ["spacetime"] * (t1 - t0 + 1)
    for cur, c in zip(range(t0, t1 + 1), calls):
        want = int(np.count_nonzero(np.abs(times - cur) <= 2 * rt))
        assert int(c[1]) == want
        assert int(c[2]) >= cur - 2 * rt and int(c[3]) <= cur + 2 * rt
        first = cur + 1 if delta else cur + 1 - 2 * rt
        assert pos[cur] == int(np.searchsorted(times, first))
        out = np.fromfile(tmp_path / f"out_{cur}.bin", OUTPOINT)
        assert out.shape[0] == 30 * 30 and np.all(out["h"] == 1.0)


@pytest.mark.parametrize("compat", [False, True])
def test_reference_caller_host_logic_on_cpu(tmp_path, compat):
    """The 2-D drop-in with a stub engine: the time slice's points go to the
    engine (canonical or reference-default call), and the OutPoints cover the
    work package clipped to the global grid, i-major (nni.cpp:836-858)."""
    lib = tmp_path / "libdnni.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-std=c99", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "native", "dnni_stub.c"), "-o", str(lib)], check=True,
                   capture_output=True, text=True)
    exe = tmp_path / "demo"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), SRC, "-o", str(exe),
                    "-L", str(tmp_path), "-ldnni", f"-Wl,-rpath,{tmp_path}"], check=True, capture_output=True,
                   text=True)
    rng = np.random.default_rng(4)
    n = 3000
    pts = np.zeros(n, POINT4D)
    pts["x"], pts["y"], pts["z"] = 100.0 + rng.uniform(0, 40, n), 200.0 + rng.uniform(0, 30, n), 5.0
    pts["t"] = np.where(np.arange(n) < 2500, 0, 1)          # the stream's next slice follows
    pin, pout, log = tmp_path / "pts.bin", tmp_path / "out.bin", tmp_path / "calls.log"
    pts.tofile(pin)
    args = [str(exe), str(pin), str(pout), "40", "30", "1.0", "100", "200", "7", "3", "45", "30", "3.0"]
    if compat:
        args += ["5", "5.0", "0", "10000"]
    r = subprocess.run(args, capture_output=True, text=True, timeout=120, env=dict(os.environ, DNNI_STUB_LOG=str(log)))
    assert r.returncode == 0, r.stderr
    call = log.read_text().split()
    assert call[0] == ("compat" if compat else "segment") and int(call[1]) == 2500
    assert "stream position 2500 of 3000" in r.stdout          # left at the next slice (nni.cpp:782-788)
    got = np.fromfile(pout, OUTPOINT)
    want = [(i + 7, j + 3) for i in range(40) for j in range(30) if i + 7 < 45 and j + 3 < 30]
    assert got.shape[0] == len(want)
    assert np.array_equal(got["i"], [w[0] for w in want]) and np.array_equal(got["j"], [w[1] for w in want])
