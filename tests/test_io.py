"""Input and output around the interpolation, on the CPU.

LAS in: files written here from the public LAS layout (independently of the
library's writer: LAS 1.2 and 1.4 headers, point formats 0, 1, 3 and 6,
variable-length records before the points) must read back record for
record, through the C ABI (raw integers, any thread count) and through the
C++ nni_io::las_reader drop-in (scaled doubles + intensity, as the
reference's libLAS reader hands them out, las_reader.inl:54-70).

Grids out: the ESRI ASCII writer must produce what the reference's outputASC
(terranni.cpp:428-488) writes for the same grid -- restated here as a
C++-stream formatter -- and the binary grid must read back bit-exact."""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REC_LEN = {0: 20, 1: 28, 3: 34, 6: 30}


def write_las_spec(path, xyz, inten, fmt, minor, scale=(0.01, 0.01, 0.001), offset=(500000.0, 4000000.0, 0.0),
                   vlr_bytes=0):
    """A LAS file per the public specification (little-endian)."""
    n = xyz.shape[0]
    hsize = 375 if minor == 4 else 227
    rec = REC_LEN[fmt]
    h = bytearray(hsize)
    h[0:4] = b"LASF"
    h[24], h[25] = 1, minor
    struct.pack_into("<HIIBH", h, 94, hsize, hsize + vlr_bytes, 1 if vlr_bytes else 0, fmt, rec)
    struct.pack_into("<I", h, 107, 0 if minor == 4 else n)
    struct.pack_into("<3d", h, 131, *scale)
    struct.pack_into("<3d", h, 155, *offset)
    lo = xyz.min(0) * np.array(scale) + np.array(offset)
    hi = xyz.max(0) * np.array(scale) + np.array(offset)
    struct.pack_into("<6d", h, 179, hi[0], lo[0], hi[1], lo[1], hi[2], lo[2])
    if minor == 4:
        struct.pack_into("<Q", h, 247, n)
    body = bytearray(n * rec)
    cls_off = 16 if fmt >= 6 else 15
    for k in range(n):
        o = k * rec
        struct.pack_into("<iiiH", body, o, int(xyz[k, 0]), int(xyz[k, 1]), int(xyz[k, 2]), int(inten[k]))
        body[o + cls_off] = 2
        body[o + rec - 1] = 0xAB        # payload the reader must skip
    with open(path, "wb") as f:
        f.write(h)
        f.write(b"\x07" * vlr_bytes)
        f.write(body)


@pytest.fixture(scope="module")
def cloud():
    rng = np.random.default_rng(5)
    n = 70_000
    xyz = np.stack([rng.integers(-2_000_000, 2_000_000, n), rng.integers(-9_000_000, 9_000_000, n),
                    rng.integers(-100_000, 300_000, n)], axis=1).astype(np.int32)
    return xyz, rng.integers(0, 65536, n).astype(np.uint16)


@pytest.mark.parametrize("fmt,minor,vlr", [(0, 2, 0), (1, 2, 54), (3, 3, 0), (6, 4, 100)])
def test_las_read_matches_the_records(tmp_path, cloud, fmt, minor, vlr):
    from terranni_b200 import engine
    xyz, inten = cloud
    p = tmp_path / f"c{fmt}.las"
    write_las_spec(p, xyz, inten, fmt, minor, vlr_bytes=vlr)
    hd = engine.las_read_header(p)
    assert (hd["version_major"], hd["version_minor"], hd["point_format"]) == (1, minor, fmt)
    assert hd["record_length"] == REC_LEN[fmt] and hd["n_points"] == xyz.shape[0]
    assert hd["scale"] == [0.01, 0.01, 0.001] and hd["offset"] == [500000.0, 4000000.0, 0.0]
    for nt in (1, 3, 0):
        got, it = engine.las_read(p, intensity=True, nthreads=nt)
        assert np.array_equal(got, xyz) and np.array_equal(it, inten)
    part = engine.las_read(p, first=12345, count=20000, nthreads=4)
    assert np.array_equal(part, xyz[12345:32345])
    with pytest.raises(engine.DnniError):
        engine.las_read(p, first=xyz.shape[0] - 10, count=11)


def test_las_write_round_trip_and_bad_files(tmp_path, cloud):
    from terranni_b200 import engine
    xyz, inten = cloud
    p = tmp_path / "w.las"
    engine.las_write(p, xyz, inten, scale=(0.01, 0.01, 0.01), offset=(1.0, 2.0, 3.0))
    hd = engine.las_read_header(p)
    assert hd["point_format"] == 0 and hd["n_points"] == xyz.shape[0]
    assert abs(hd["min"][0] - (xyz[:, 0].min() * 0.01 + 1.0)) < 1e-6
    got, it = engine.las_read(p, intensity=True)
    assert np.array_equal(got, xyz) and np.array_equal(it, inten)
    bad = tmp_path / "bad.las"
    bad.write_bytes(b"NOPE" + bytes(400))
    with pytest.raises(engine.DnniError):
        engine.las_read_header(bad)
    laz = bytearray(p.read_bytes())
    laz[104] |= 0x80                                   # compressed point data
    (tmp_path / "c.laz").write_bytes(bytes(laz))
    with pytest.raises(engine.DnniError):
        engine.las_read_header(tmp_path / "c.laz")


def test_cpp_las_reader_dropin(tmp_path, cloud):
    from terranni_b200 import engine
    xyz, inten = cloud
    p = tmp_path / "r.las"
    write_las_spec(p, xyz[:5000], inten[:5000], 3, 2, vlr_bytes=54)
    src = tmp_path / "rd.cpp"
    src.write_text(r'''
#include <cstdio>
#include <nni/nni.h>
#include <nni_io/las_reader.h>
int main(int, char** argv) {
    nni_io::las_reader<nni::Point4D, double> r;
    r.open(argv[1]);
    nni::Point4D p;
    long n = 0;
    FILE* o = std::fopen(argv[2], "wb");
    for (int pass = 0; pass < 2; ++pass) {          // reset() starts over
        while (r.next_point(p)) {
            if (pass == 1) { std::fwrite(p.p, sizeof(double), 3, o); std::fwrite(&p.t, sizeof(int), 1, o); }
            ++n;
        }
        r.reset();
    }
    std::fclose(o);
    r.close();
    std::printf("%ld %llu\n", n, (unsigned long long)r.get_header().n_points);
    return r.next_point(p) ? 1 : 0;                  // closed: no more points
}
''')
    exe = tmp_path / "rd"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", os.path.join(ROOT, "terranni_b200"), "-ldnni",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'terranni_b200')}"], check=True, capture_output=True)
    out = tmp_path / "pts.bin"
    r = subprocess.run([str(exe), str(p), str(out)], capture_output=True, text=True, check=True)
    assert r.stdout.split() == ["10000", "5000"]
    rec = np.fromfile(out, np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("t", "<i4")]))
    assert np.array_equal(rec["x"], xyz[:5000, 0] * 0.01 + 500000.0)
    assert np.array_equal(rec["y"], xyz[:5000, 1] * 0.01 + 4000000.0)
    assert np.array_equal(rec["z"], xyz[:5000, 2] * 0.001 + 0.0)
    assert np.array_equal(rec["t"], inten[:5000].astype(np.int32))


def _asc_reference(h, xll, yll, cs):
    """outputASC's text for a row-major grid (row 0 = lowest y): a C++
    stream prints floats with 6 significant digits, i.e. printf's %g."""
    nrows, ncols = h.shape
    out = [f"NROWS {nrows}\n", f"NCOLS {ncols}\n", f"XLLCORNER {xll:.10g}\n", f"YLLCORNER {yll:.10g}\n",
           f"CELLSIZE {cs:.10g}\n", "NODATA_VALUE -9999\n"]
    for j in range(nrows - 1, -1, -1):
        out.append("".join("%g " % float(v) for v in h[j]) + "\n")
    return "".join(out)


def test_ascii_grid_as_output_asc(tmp_path):
    from terranni_b200 import engine
    rng = np.random.default_rng(2)
    h = (rng.random((150, 97)) * 300).astype(np.float32)
    h[3, 5] = np.float32(-9999.0)
    h[7, 1] = np.float32(1e-7)
    h[0, 0] = np.float32(123456789.0)
    p = tmp_path / "g.asc"
    for nt in (1, 5):
        engine.write_asc(p, h, 500000.5, 4000000.25, 1.0, nthreads=nt)
        assert p.read_text() == _asc_reference(h, 500000.5, 4000000.25, 1.0)


def test_binary_grid_round_trip(tmp_path):
    from terranni_b200 import engine
    h = np.random.default_rng(3).random((33, 44)).astype(np.float32)
    p = tmp_path / "g.bin"
    engine.write_grid_bin(p, h, 10.0, 20.0, 0.5, -9999.0)
    raw = p.read_bytes()
    assert raw[:8] == b"DNNIGRD1"
    ncols, nrows = struct.unpack_from("<ii", raw, 8)
    xll, yll, cs = struct.unpack_from("<3d", raw, 16)
    (nod,) = struct.unpack_from("<f", raw, 40)
    assert (ncols, nrows, xll, yll, cs, nod) == (44, 33, 10.0, 20.0, 0.5, -9999.0)
    assert np.array_equal(np.frombuffer(raw, np.float32, offset=64).reshape(33, 44), h)
