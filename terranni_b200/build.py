"""Build recipe for the engine's native libraries (in-tree, sm_100a only).

  libdnni.so        CUDA engine + C ABI (include/dnni.h) + C++ shim (include/nni/nni.h)
  libdnni_synth.so  seeded synthetic point-cloud generator (host C, OpenMP)

Run ``python -m terranni_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
OBJ = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
           "-I" + os.path.join(ROOT, "include")]

CUDA_SOURCES = ["dnni_engine.cu"]
CXX_SOURCES = ["dnni_io.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include"), os.path.join(ROOT, "include", "nni"),
              os.path.join(ROOT, "include", "nni_io")):
        if os.path.isdir(d):
            out += [os.path.join(d, f) for f in os.listdir(d)
                    if f.endswith((".cu", ".cuh", ".h", ".hpp", ".cpp", ".c", ".inl"))]
    return out


def build(force: bool = False, verbose: bool = False) -> dict:
    os.makedirs(OBJ, exist_ok=True)
    deps = _deps()
    lib = os.path.join(HERE, "libdnni.so")
    if force or _stale(lib, deps):
        objs = []
        for src in CUDA_SOURCES:
            o = os.path.join(OBJ, src + ".o")
            cmd = [NVCC] + ARCH + NVFLAGS + ["-c", os.path.join(CSRC, src), "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
            objs.append(o)
        for src in CXX_SOURCES:
            o = os.path.join(OBJ, src + ".o")
            _run([NVCC] + NVFLAGS + ["-x", "c++", "-c", os.path.join(CSRC, src), "-o", o])
            objs.append(o)
        _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"])
    synth = os.path.join(HERE, "libdnni_synth.so")
    src = os.path.join(CSRC, "synth.c")
    if force or _stale(synth, [src]):
        _run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-o", synth, src, "-lm"])
    return {"libdnni": lib, "libdnni_synth": synth}


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
