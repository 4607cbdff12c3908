"""The C ABI library loads and exports every symbol its headers declare."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    return sorted(set(re.findall(r"\b(dnni_[a-z0-9_]+)\s*\(", src)))


def test_libdnni_exports_every_declared_symbol():
    from terranni_b200 import engine
    L = engine.lib()
    names = declared("dnni.h")
    assert len(names) >= 11
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) <= set(engine.exported_symbols())


def test_version():
    from terranni_b200 import engine
    assert engine.lib().dnni_version() == 10000


def test_init_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    from terranni_b200 import engine
    h = ctypes.c_void_p()
    assert engine.lib().dnni_init(None, ctypes.byref(h)) == 4   # DNNI_E_CUDA
    assert not h.value


def test_null_arguments_rejected():
    from terranni_b200 import engine
    L = engine.lib()
    assert L.dnni_measure_peaks(0, None) == 1
    assert L.dnni_init(None, None) == 1
    assert L.dnni_destroy(None) == 1
    assert L.dnni_last_error(None) == b"context is NULL"


def test_synth_is_seeded_and_thread_independent():
    from terranni_b200 import synth
    a, la = synth.generate(42, 20000, 300.0, 200.0, nlakes=3, lake_rmin=10, lake_rmax=40, nthreads=1)
    b, lb = synth.generate(42, 20000, 300.0, 200.0, nlakes=3, lake_rmin=10, lake_rmax=40, nthreads=4)
    assert np.array_equal(a, b) and np.array_equal(la, lb)
    assert a[:, 0].min() >= 0 and a[:, 0].max() < 30000 and a[:, 1].max() < 20000
    # no point inside a lake
    for cx, cy, r in la:
        d2 = (a[:, 0] * 0.01 - cx) ** 2 + (a[:, 1] * 0.01 - cy) ** 2
        assert (d2 >= (r - 0.01) ** 2).all()
    c, _ = synth.generate(43, 20000, 300.0, 200.0, nlakes=3, lake_rmin=10, lake_rmax=40)
    assert not np.array_equal(a, c)


def test_sinusoid_workload_shape():
    from terranni_b200 import synth
    w = synth.config1()
    xyz = w["xyz"]
    assert xyz.shape == (200000, 3)
    assert xyz[:, :2].min() >= 0 and xyz[:, :2].max() < 51200
    z = xyz[:, 2] * 0.01
    assert -80.5 < z.min() < 0 < z.max() < 80.5


def test_header_is_plain_c_and_links(tmp_path):
    # a C99 translation unit (what cgo, JNI or ctypes bindings would see)
    # takes the address of every declared function and links against the
    # library
    import subprocess
    names = declared("dnni.h")
    src = tmp_path / "abi.c"
    src.write_text("#include <stdio.h>\n#include \"dnni.h\"\ntypedef void (*fn_t)(void);\nint main(void) {\n"
                   "    fn_t fns[] = {\n" + "".join(f"        (fn_t)&{n},\n" for n in names) + "    };\n"
                   "    printf(\"%d\\n\", (int)(sizeof(fns) / sizeof(fns[0])));\n"
                   "    return dnni_version() == 10000 ? 0 : 1;\n}\n")
    exe = tmp_path / "abi"
    lib = os.path.join(ROOT, "terranni_b200")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", lib, "-ldnni", f"-Wl,-rpath,{lib}"], check=True,
                   capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and int(r.stdout) == len(names)


def test_new_entry_points_reject_null_arguments():
    from terranni_b200 import engine
    L = engine.lib()
    for name in ("dnni_interpolate_spacetime", "dnni_interpolate_spacetime_device", "dnni_interpolate_compat",
                 "dnni_interpolate_compat_device"):
        f = getattr(L, name)
        args = [0 if t in (ctypes.c_int64, ctypes.c_int32, ctypes.c_int) else None for t in f.argtypes]
        assert f(*args) == 1, name                 # NULL context: DNNI_E_INVAL


def test_pinned_host_allocation_arguments():
    # dnni_host_alloc / dnni_host_free: NULL handling, and without a device a
    # clean DNNI_E_NOMEM with NULL
    import torch
    from terranni_b200 import engine
    L = engine.lib()
    assert L.dnni_host_alloc(16, None) == 1
    assert L.dnni_host_free(None) == 0
    if torch.cuda.is_available():
        return
    p = ctypes.c_void_p()
    assert L.dnni_host_alloc(1 << 20, ctypes.byref(p)) == 2 and not p.value


@pytest.mark.gpu
def test_pinned_host_allocation():
    from terranni_b200 import engine
    L = engine.lib()
    p = ctypes.c_void_p()
    assert L.dnni_host_alloc(1 << 20, ctypes.byref(p)) == 0 and p.value
    buf = (ctypes.c_uint8 * (1 << 20)).from_address(p.value)
    buf[0], buf[(1 << 20) - 1] = 7, 9
    assert buf[0] == 7 and buf[(1 << 20) - 1] == 9
    assert L.dnni_host_free(p) == 0


def test_python_binding_layouts_match_the_header(tmp_path):
    # every ctypes structure of the binding has the size and field offsets of
    # the C struct it stands for (a C99 program prints offsetof/sizeof)
    import subprocess
    from terranni_b200 import engine
    pairs = {"Settings": "dnni_settings", "WorkPackage": "dnni_workpackage", "Stats": "dnni_stats",
             "Tile": "dnni_tile", "BatchOptions": "dnni_batch_options", "Segment": "dnni_segment",
             "SegmentStats": "dnni_segment_stats", "ServerOptions": "dnni_server_options",
             "Request": "dnni_request", "RequestResult": "dnni_request_result", "ServerStats": "dnni_server_stats",
             "LasHeader": "dnni_las_header", "CompatSettings": "dnni_compat_settings", "StOptions": "dnni_st_options",
             "CompatWP": "dnni_compat_wp", "Peaks": "dnni_peaks", "TuneTrial": "dnni_tune_trial",
             "TuneReport": "dnni_tune_report"}
    lines = ["#include <stdio.h>", "#include <stddef.h>", "#include \"dnni.h\"", "int main(void) {"]
    want = []
    for py, c in pairs.items():
        cls = getattr(engine, py)
        lines.append(f"    printf(\"%zu\\n\", sizeof({c}));")
        want.append((f"sizeof {c}", ctypes.sizeof(cls)))
        for name, *_ in cls._fields_:
            lines.append(f"    printf(\"%zu\\n\", offsetof({c}, {name}));")
            want.append((f"{c}.{name}", getattr(cls, name).offset))
    lines.append("    return 0;\n}\n")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert len(got) == len(want)
    bad = [(k, g, w) for (k, w), g in zip(want, got) if g != w]
    assert not bad, bad
